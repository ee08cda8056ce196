"""Batched creature engine (include/kraken_batch.h) from Python.

    eng = BatchEngine(maps, capacity=16384, obs_ring=0, control="stream")
    eng.spawn(0, arms, segs, map_id, x, y, angle, horizon, seed)
    eng.run(200)                      # one persistent launch, <= 200 steps each
    state = eng.read_state(0, 16)     # bodies (px py vx vy ang av), grips, steps

Every creature behaves like a one-creature gpuworld world driven by the
reference's hybrid loop (readProprio -> controls -> applyControl reflex ->
step, src/sim/gputrain.js:72-128), with the reflex and the proprioception on
the device.  There is no CPU fallback: without the CUDA library every call
raises.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native

MAX_ARMS = 8
MAX_SEGS = 9
MAX_BODIES = 1 + MAX_ARMS * MAX_SEGS
OBS_STRIDE = 56
CTRL_STRIDE = MAX_ARMS * (MAX_SEGS + 1)
POLICY_HIDDEN = 64
CONTROL_MODES = {"stream": 0, "buffer": 1, "policy": 2, "net": 3}
# KR_CTRL_NET: net.js HIDDEN, echo.js ECHO_RAYS, lights per map, read strides
NET_HIDDEN = 24
NET_RAYS = 12
NET_MAX_LIGHTS = 8
NET_IN_STRIDE = 128
NET_OUT_STRIDE = 32


def net_inputs(arms):
    """Input size of the reference net for an arms-armed body (105 at 6 arms)."""
    return 10 * arms + 45


def net_outputs(arms):
    """Outputs of the reference net: tone, 3 per arm, echo (20 at 6 arms)."""
    return 3 * arms + 2


def net_param_count(arms):
    """net.js weightCount (3,644 at 6 arms)."""
    ni, no, h = net_inputs(arms), net_outputs(arms), NET_HIDDEN
    return ni * h + h + h * h + h + h * no + no
# the reference's fitness metrics (postStep, src/sim/core.js:297-356) and score
# (src/sim/fitness.js:115-172), in kr_batch_read_metrics order
METRIC_FIELDS = ("score", "steps", "pathLen", "maxDisplacement", "spawnReach", "angularAccum",
                 "forwardProg", "gripPullProg", "anchoredSteps", "freeMove", "energySpent",
                 "gripCycles", "strides", "attachEvents", "x", "y")
METRIC_WORDS = len(METRIC_FIELDS)

_F32P = C.POINTER(C.c_float)
_F64P = C.POINTER(C.c_double)
_I32P = C.POINTER(C.c_int32)
_I64P = C.POINTER(C.c_int64)
_U32P = C.POINTER(C.c_uint32)


class BatchDesc(C.Structure):
    _fields_ = [("solver", _native.SolverParams), ("n_maps", C.c_int32),
                ("rects", _F32P), ("map_rect_off", _I32P), ("capacity", C.c_int32),
                ("obs_ring", C.c_int32), ("grip_slip_max", C.c_double),
                ("grip_cooldown", C.c_double), ("control_mode", C.c_int32),
                ("control_period", C.c_int32), ("lights", _F64P), ("map_light_off", _I32P),
                ("map_size", _F64P)]


_bound = False


def _lib():
    global _bound
    L = _native.lib()
    if _bound:
        return L
    vp, i32 = C.c_void_p, C.c_int32
    sigs = {
        "kr_batch_create": (C.c_int, [C.POINTER(BatchDesc), C.POINTER(vp)]),
        "kr_batch_spawn": (C.c_int, [vp, i32, i32, _I32P, _I32P, _I32P, _F64P, _F64P, _F64P,
                                     _I32P, _U32P, _F32P]),
        "kr_batch_set_controls": (C.c_int, [vp, _F32P]),
        "kr_batch_set_policy": (C.c_int, [vp, _F32P, i32, i32, _I32P]),
        "kr_batch_set_net": (C.c_int, [vp, _F32P, i32, i32, _I32P]),
        "kr_batch_read_net": (C.c_int, [vp, i32, i32, _F32P, _F32P]),
        "kr_batch_run": (C.c_int, [vp, i32]),
        "kr_batch_run_graph": (C.c_int, [vp, i32, i32, i32]),
        "kr_batch_run_launches": (C.c_int, [vp, i32, i32]),
        "kr_batch_live": (C.c_int, [vp, _I32P]),
        "kr_batch_read_state": (C.c_int, [vp, i32, i32, _F32P, _F32P, _I32P]),
        "kr_batch_read_obs": (C.c_int, [vp, i32, i32, _F32P]),
        "kr_batch_read_fitness": (C.c_int, [vp, i32, i32, _F64P]),
        "kr_batch_read_controls": (C.c_int, [vp, i32, i32, _F32P]),
        "kr_batch_read_metrics": (C.c_int, [vp, i32, i32, _F64P]),
        "kr_batch_set_launch": (C.c_int, [vp, i32, i32, i32]),
        "kr_batch_get_launch": (C.c_int, [vp, _I32P, _I32P, _I32P, _I32P]),
        "kr_batch_autotune": (C.c_int, [vp, i32, _I32P, _I32P, _I32P, _F32P]),
        "kr_batch_set_unroll": (C.c_int, [vp, i32]),
        "kr_batch_get_unroll": (C.c_int, [vp, _I32P]),
        "kr_batch_last_ms": (C.c_int, [vp, _F32P]),
        "kr_batch_set_slice": (C.c_int, [vp, C.c_float]),
        "kr_batch_last_slices": (C.c_int, [vp, _I32P, _I32P, _I64P]),
        "kr_batch_sync": (C.c_int, [vp]),
        "kr_batch_set_stream": (C.c_int, [vp, vp]),
        "kr_batch_destroy": (None, [vp]),
        "kr_batch_last_error": (C.c_char_p, [vp]),
        "kr_batch_snapshot": (C.c_int, [vp]),
        "kr_batch_restore": (C.c_int, [vp]),
        "kr_probe_fp32_rate": (C.c_int, [_F64P]),
        "kr_probe_sincos": (C.c_int, [_F32P, i32, _F32P, _F32P]),
        "kr_probe_wrap": (C.c_int, [_F64P, i32, _F64P]),
    }
    for name, (res, args) in sigs.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _bound = True
    return L


def _check(rc, handle):
    if rc != _native.KR_OK:
        msg = _lib().kr_batch_last_error(handle)
        raise _native.KrError(rc, msg.decode() if msg else f"status {rc}")


def _arr(a, dtype):
    return np.ascontiguousarray(np.asarray(a), dtype=dtype)


class BatchEngine:
    """One batched engine handle (kr_batch)."""

    def __init__(self, maps, capacity, obs_ring=0, control="stream", control_period=6,
                 substeps=2, iterations=4, h=1 / 120, lin_drag=3.0, ang_drag=3.0,
                 max_speed=360.0, max_ang_speed=18.0, grip_slip_max=150.0, grip_cooldown=0.05,
                 lights=None, map_size=(1440.0, 810.0)):
        """maps: per map an (n, 4) array of rects x y w h.  control="net":
        lights, per map an (n, 6) array x y r ir ph sp (or None: no lights),
        and map_size (width, height) of every map, the lights' clamp."""
        L = _lib()
        rect_list = [np.asarray(m, dtype=np.float32).reshape(-1, 4) for m in maps]
        off = np.zeros(len(rect_list) + 1, dtype=np.int32)
        for i, r in enumerate(rect_list):
            off[i + 1] = off[i] + len(r)
        rects = np.ascontiguousarray(np.concatenate(rect_list) if rect_list else
                                     np.zeros((0, 4), np.float32), dtype=np.float32)
        self.capacity = int(capacity)
        self.obs_ring = int(obs_ring)
        self.control = control
        d = BatchDesc(_native.SolverParams(h, substeps, iterations, lin_drag, ang_drag, max_speed,
                                           max_ang_speed),
                      len(rect_list), rects.ctypes.data_as(_F32P), off.ctypes.data_as(_I32P),
                      self.capacity, self.obs_ring, grip_slip_max, grip_cooldown,
                      CONTROL_MODES[control], control_period)
        if control == "net" and lights is not None:
            lv = [np.asarray(l, dtype=np.float64).reshape(-1, 6) for l in lights]
            if len(lv) != len(rect_list):
                raise ValueError("one light array per map")
            loff = np.zeros(len(lv) + 1, dtype=np.int32)
            for i, l in enumerate(lv):
                loff[i + 1] = loff[i] + len(l)
            self._lights = np.ascontiguousarray(np.concatenate(lv) if lv else np.zeros((0, 6)))
            self._light_off = loff
            self._map_size = np.ascontiguousarray(np.tile(np.asarray(map_size, np.float64),
                                                          (len(lv), 1)))
            d.lights = self._lights.ctypes.data_as(_F64P)
            d.map_light_off = self._light_off.ctypes.data_as(_I32P)
            d.map_size = self._map_size.ctypes.data_as(_F64P)
        self.h = C.c_void_p()
        rc = L.kr_batch_create(C.byref(d), C.byref(self.h))
        _check(rc, None)
        self.arms = np.zeros(self.capacity, dtype=np.int32)
        self.segs = np.zeros(self.capacity, dtype=np.int32)

    def close(self):
        if getattr(self, "h", None) and self.h.value:
            _lib().kr_batch_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def spawn(self, first, arms, segs, map_id, x, y, angle, horizon, seed=None, tone=None):
        n = len(x)
        arms, segs = _arr(arms, np.int32), _arr(segs, np.int32)
        map_id, horizon = _arr(map_id, np.int32), _arr(horizon, np.int32)
        x, y, angle = _arr(x, np.float64), _arr(y, np.float64), _arr(angle, np.float64)
        seed = _arr(np.arange(first, first + n) if seed is None else seed, np.uint32)
        tone = _arr(np.full(n, 0.5) if tone is None else tone, np.float32)
        rc = _lib().kr_batch_spawn(self.h, first, n, arms.ctypes.data_as(_I32P),
                                   segs.ctypes.data_as(_I32P), map_id.ctypes.data_as(_I32P),
                                   x.ctypes.data_as(_F64P), y.ctypes.data_as(_F64P),
                                   angle.ctypes.data_as(_F64P), horizon.ctypes.data_as(_I32P),
                                   seed.ctypes.data_as(_U32P), tone.ctypes.data_as(_F32P))
        _check(rc, self.h)
        self.arms[first:first + n] = arms
        self.segs[first:first + n] = segs

    def set_controls(self, controls):
        c = _arr(controls, np.float32).reshape(self.capacity, CTRL_STRIDE)
        _check(_lib().kr_batch_set_controls(self.h, c.ctypes.data_as(_F32P)), self.h)

    def set_policy(self, weights, slot_individual):
        w = _arr(weights, np.float32)
        w = w.reshape(w.shape[0], -1)
        idx = _arr(slot_individual, np.int32)
        _check(_lib().kr_batch_set_policy(self.h, w.ctypes.data_as(_F32P), w.shape[0], w.shape[1],
                                          idx.ctypes.data_as(_I32P)), self.h)

    def set_net(self, genomes, slot_individual):
        """control="net": genomes (n_individuals, n) f32, each row in net.js's
        layout for its slots' arm count (first net_param_count(arms) floats
        read, n at least that); slot s uses genome slot_individual[s]."""
        g = _arr(genomes, np.float32)
        g = g.reshape(g.shape[0], -1)
        idx = _arr(slot_individual, np.int32)
        _check(_lib().kr_batch_set_net(self.h, g.ctypes.data_as(_F32P), g.shape[0], g.shape[1],
                                       idx.ctypes.data_as(_I32P)), self.h)

    def read_net(self, first=0, n=None):
        """control="net": (inputs (n, NET_IN_STRIDE), outputs (n, NET_OUT_STRIDE))
        f32 of each slot's last env step (net_inputs / net_outputs used)."""
        n = self.capacity - first if n is None else n
        x = np.zeros((n, NET_IN_STRIDE), dtype=np.float32)
        o = np.zeros((n, NET_OUT_STRIDE), dtype=np.float32)
        _check(_lib().kr_batch_read_net(self.h, first, n, x.ctypes.data_as(_F32P),
                                        o.ctypes.data_as(_F32P)), self.h)
        return x, o

    def snapshot(self):
        _check(_lib().kr_batch_snapshot(self.h), self.h)

    def restore(self):
        _check(_lib().kr_batch_restore(self.h), self.h)

    def set_launch(self, warps_per_cta, ctas_per_sm=0, lanes_per_creature=32):
        """Launch shape: G lanes per creature (32, 16 or 8; 0: the automatic
        shape of every launch again), warps per CTA, CTAs per SM (0: 16 /
        warps).  Results do not depend on it."""
        _check(_lib().kr_batch_set_launch(self.h, lanes_per_creature, warps_per_cta, ctas_per_sm),
               self.h)

    def set_unroll(self, substep_unroll):
        """Unroll factor of the kernel's substep loop (1 or 2); results do
        not depend on it."""
        _check(_lib().kr_batch_set_unroll(self.h, substep_unroll), self.h)

    def autotune(self, steps=64):
        """Time every candidate launch shape (lanes, warps, CTAs per SM,
        substep unroll) on `steps` env steps of the live slots (state put back
        after each trial), keep the fastest; returns (lanes_per_creature,
        warps_per_cta, ctas_per_sm, ms) -- the unroll is in get_launch()."""
        v = [C.c_int32() for _ in range(3)]
        ms = C.c_float()
        _check(_lib().kr_batch_autotune(self.h, steps, *[C.byref(x) for x in v], C.byref(ms)), self.h)
        return v[0].value, v[1].value, v[2].value, ms.value

    def get_launch(self):
        v = [C.c_int32() for _ in range(5)]
        _check(_lib().kr_batch_get_launch(self.h, *[C.byref(x) for x in v[:4]]), self.h)
        _check(_lib().kr_batch_get_unroll(self.h, C.byref(v[4])), self.h)
        return {"lanes_per_creature": v[0].value, "warps_per_cta": v[1].value,
                "ctas_per_sm": v[2].value, "smem_bytes": v[3].value, "substep_unroll": v[4].value}

    def run(self, max_steps):
        _check(_lib().kr_batch_run(self.h, max_steps), self.h)

    def set_slice(self, slice_ms):
        """Time slices (ms) for runs that take every live slot to its horizon:
        preemptible launches, the creatures regrouped between them (0: one
        launch).  Results do not depend on it."""
        _check(_lib().kr_batch_set_slice(self.h, float(slice_ms)), self.h)

    def last_slices(self) -> int:
        return self.last_run_launches()[0]

    def last_run_launches(self):
        """(slices, kernels launched, creatures launched summed over the
        slices) of the last run."""
        n, k, c = C.c_int32(), C.c_int32(), C.c_int64()
        _check(_lib().kr_batch_last_slices(self.h, C.byref(n), C.byref(k), C.byref(c)), self.h)
        return n.value, k.value, c.value

    def run_launches(self, steps_per_launch, launches):
        _check(_lib().kr_batch_run_launches(self.h, steps_per_launch, launches), self.h)

    def set_stream(self, stream_ptr):
        _check(_lib().kr_batch_set_stream(self.h, C.c_void_p(stream_ptr)), self.h)

    def run_graph(self, max_steps, launches, replays=1):
        _check(_lib().kr_batch_run_graph(self.h, max_steps, launches, replays), self.h)

    def sync(self):
        _check(_lib().kr_batch_sync(self.h), self.h)

    def last_ms(self) -> float:
        ms = C.c_float()
        _check(_lib().kr_batch_last_ms(self.h, C.byref(ms)), self.h)
        return ms.value

    def live(self) -> int:
        n = C.c_int32()
        _check(_lib().kr_batch_live(self.h, C.byref(n)), self.h)
        return n.value

    def read_state(self, first=0, n=None):
        n = self.capacity - first if n is None else n
        bodies = np.zeros((n, MAX_BODIES, 6), dtype=np.float32)
        grips = np.zeros((n, MAX_ARMS, 4), dtype=np.float32)
        steps = np.zeros(n, dtype=np.int32)
        _check(_lib().kr_batch_read_state(self.h, first, n, bodies.ctypes.data_as(_F32P),
                                          grips.ctypes.data_as(_F32P),
                                          steps.ctypes.data_as(_I32P)), self.h)
        return {"px": bodies[..., 0], "py": bodies[..., 1], "vx": bodies[..., 2],
                "vy": bodies[..., 3], "ang": bodies[..., 4], "av": bodies[..., 5],
                "grips": grips, "steps": steps}

    def read_obs(self, first=0, n=None):
        n = self.capacity - first if n is None else n
        out = np.zeros((n, self.obs_ring, OBS_STRIDE), dtype=np.float32)
        _check(_lib().kr_batch_read_obs(self.h, first, n, out.ctypes.data_as(_F32P)), self.h)
        return out

    def read_controls(self, first=0, n=None):
        """Controls of each slot's last env step: (n, CTRL_STRIDE) f32, motor
        controls (arm-major, shoulder first) then adhesion values."""
        n = self.capacity - first if n is None else n
        out = np.zeros((n, CTRL_STRIDE), dtype=np.float32)
        _check(_lib().kr_batch_read_controls(self.h, first, n, out.ctypes.data_as(_F32P)), self.h)
        return out

    def read_metrics(self, first=0, n=None):
        """(n, METRIC_WORDS) f64: the reference's score and postStep metrics
        of each slot (METRIC_FIELDS order)."""
        n = self.capacity - first if n is None else n
        out = np.zeros((n, METRIC_WORDS), dtype=np.float64)
        _check(_lib().kr_batch_read_metrics(self.h, first, n, out.ctypes.data_as(_F64P)), self.h)
        return out

    def read_fitness(self, first=0, n=None):
        n = self.capacity - first if n is None else n
        out = np.zeros((n, 4), dtype=np.float64)
        _check(_lib().kr_batch_read_fitness(self.h, first, n, out.ctypes.data_as(_F64P)), self.h)
        return out


def policy_params(arms=6, segs=7) -> int:
    """Parameter count of the fused controller for an arms x segs body."""
    n_in, n_out = 6 * arms + 6, arms * segs + arms
    return POLICY_HIDDEN * (n_in + 1) + n_out * (POLICY_HIDDEN + 1)


def probe_fp32_rate() -> float:
    """Measured dependent-free f32 FMA instructions per second of the device."""
    r = C.c_double()
    _check(_lib().kr_probe_fp32_rate(C.byref(r)), None)
    return r.value


def probe_wrap(d):
    """readProprio's atan2(sin d, cos d) of f64 angle differences as the
    device evaluates it (d wrapped into (-pi, pi])."""
    d = np.ascontiguousarray(d, dtype=np.float64)
    out = np.zeros_like(d)
    _check(_lib().kr_probe_wrap(d.ctypes.data_as(_F64P), len(d), out.ctypes.data_as(_F64P)), None)
    return out


def probe_sincos(x):
    """The solver's device sin / cos of f32 angles (each the f64 value
    rounded once to f32): (sin, cos) arrays."""
    x = np.ascontiguousarray(x, dtype=np.float32)
    s = np.zeros_like(x)
    c = np.zeros_like(x)
    _check(_lib().kr_probe_sincos(x.ctypes.data_as(_F32P), len(x), s.ctypes.data_as(_F32P),
                                  c.ctypes.data_as(_F32P)), None)
    return s, c
