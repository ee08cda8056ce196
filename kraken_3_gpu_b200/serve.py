"""Rollout server (include/kraken_serve.h) from Python.

    srv = Server(maps, hbm_budget=8 << 30, max_slots=16384, chunk_steps=32)
    rid = srv.submit(population=64, horizon=600, arms=6, segs=7, map_id=0,
                     x=400, y=300, angle=0.0, theta=theta, sigma=0.02, seed=7)
    srv.drain()
    res = srv.result(rid)        # {"results": (64, 4) f64, "arrival", "admitted", "completed"}

Requests are mirrored ES populations (individual 2k: theta + sigma*eps_k,
2k+1: theta - sigma*eps_k, eps drawn on the device from the seed) of one body
shape on one map; without theta the individuals follow control streams from
the seed.  Requests arriving while others run are admitted into free slots
between rounds and share the GPU's launches (continuous batching); the HBM
budget fixes the slot count.  There is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native
from .batch import net_param_count, policy_params  # noqa: F401  (parameter counts of a body's controllers)

from .batch import METRIC_FIELDS as RESULT_FIELDS  # noqa: E402
RESULT_WORDS = len(RESULT_FIELDS)

_F32P = C.POINTER(C.c_float)
_F64P = C.POINTER(C.c_double)
_I32P = C.POINTER(C.c_int32)
_I64P = C.POINTER(C.c_int64)


class ServerDesc(C.Structure):
    _fields_ = [("solver", _native.SolverParams), ("n_maps", C.c_int32), ("rects", _F32P),
                ("map_rect_off", _I32P), ("hbm_budget_bytes", C.c_uint64), ("max_slots", C.c_int32),
                ("obs_ring", C.c_int32), ("chunk_steps", C.c_int32), ("policy", C.c_int32),
                ("lanes_per_creature", C.c_int32), ("warps_per_cta", C.c_int32),
                ("ctas_per_sm", C.c_int32), ("grip_slip_max", C.c_double),
                ("grip_cooldown", C.c_double), ("net", C.c_int32), ("lights", _F64P),
                ("map_light_off", _I32P), ("map_size", _F64P), ("slice_ms", C.c_double)]


class Request(C.Structure):
    _fields_ = [("population", C.c_int32), ("horizon", C.c_int32), ("arms", C.c_int32),
                ("segs", C.c_int32), ("map_id", C.c_int32), ("x", C.c_double), ("y", C.c_double),
                ("angle", C.c_double), ("xs", _F64P), ("ys", _F64P), ("angles", _F64P),
                ("control_seeds", C.POINTER(C.c_uint32)),
                ("tone", C.c_float), ("theta", _F32P), ("n_params", C.c_int32),
                ("sigma", C.c_float), ("seed", C.c_uint64), ("arrival", C.c_double),
                ("first_individual", C.c_int32)]


class _RequestRaw(C.Structure):
    """kr_request with the pointers as integers (same layout), for numpy."""
    _fields_ = [(n, C.c_uint64 if t in (_F32P, _F64P, C.POINTER(C.c_uint32)) else t)
                for n, t in Request._fields_]


REQUEST_DTYPE = np.dtype(_RequestRaw)
assert REQUEST_DTYPE.itemsize == C.sizeof(Request)


class Stats(C.Structure):
    _fields_ = [("capacity", C.c_int32), ("partition_capacity", C.c_int32), ("live", C.c_int32),
                ("queued", C.c_int32), ("submitted", C.c_int64), ("admitted", C.c_int64),
                ("completed", C.c_int64), ("rounds", C.c_int64), ("creature_steps", C.c_double),
                ("device_ms", C.c_double), ("bytes_per_slot", C.c_uint64), ("device_bytes", C.c_uint64),
                ("h2d_bytes", C.c_uint64), ("d2h_bytes", C.c_uint64), ("host_gap_ms", C.c_double)]


_bound = False


def _lib():
    global _bound
    L = _native.lib()
    if _bound:
        return L
    vp, i32 = C.c_void_p, C.c_int32
    sigs = {
        "kr_server_plan": (C.c_int, [C.POINTER(ServerDesc), _I32P, C.POINTER(C.c_uint64)]),
        "kr_server_create": (C.c_int, [C.POINTER(ServerDesc), C.POINTER(vp)]),
        "kr_server_now": (C.c_double, [vp]),
        "kr_server_submit": (C.c_int, [vp, C.POINTER(Request), _I64P]),
        "kr_server_pump": (C.c_int, [vp, _I32P]),
        "kr_server_submit_batch": (C.c_int, [vp, vp, i32, _I64P, _I32P]),
        "kr_server_result_batch": (C.c_int, [vp, _I64P, i32, _F64P, _F64P, i32]),
        "kr_server_drain": (C.c_int, [vp]),
        "kr_server_poll": (C.c_int, [vp, _I64P, i32, _I32P]),
        "kr_server_result": (C.c_int, [vp, C.c_int64, _F64P, _F64P]),
        "kr_server_release": (C.c_int, [vp, C.c_int64]),
        "kr_server_get_stats": (C.c_int, [vp, C.POINTER(Stats)]),
        "kr_server_destroy": (None, [vp]),
        "kr_server_last_error": (C.c_char_p, [vp]),
        "kr_policy_eps": (C.c_int, [C.c_uint64, i32, i32, _F32P]),
    }
    for name, (res, args) in sigs.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _bound = True
    return L


def _check(rc, h):
    if rc != 0:
        msg = _lib().kr_server_last_error(h)
        raise _native.KrError(rc, (msg or b"").decode() or f"kraken server error {rc}")


def _desc(maps, hbm_budget, max_slots, obs_ring, chunk_steps, policy, lanes, warps, ctas,
          substeps, iterations, h, lin_drag, ang_drag, max_speed, max_ang_speed, grip_slip_max,
          grip_cooldown, net, lights, map_size, slice_ms):
    rect_list = [np.asarray(m, dtype=np.float32).reshape(-1, 4) for m in maps]
    off = np.zeros(len(rect_list) + 1, dtype=np.int32)
    for i, r in enumerate(rect_list):
        off[i + 1] = off[i] + len(r)
    rects = np.ascontiguousarray(np.concatenate(rect_list) if rect_list else
                                 np.zeros((0, 4), np.float32), dtype=np.float32)
    d = ServerDesc(_native.SolverParams(h, substeps, iterations, lin_drag, ang_drag, max_speed,
                                        max_ang_speed),
                   len(rect_list), rects.ctypes.data_as(_F32P), off.ctypes.data_as(_I32P),
                   int(hbm_budget), int(max_slots), int(obs_ring), int(chunk_steps), int(policy),
                   int(lanes), int(warps), int(ctas), grip_slip_max, grip_cooldown)
    d.slice_ms = float(slice_ms)
    keep = [rects, off]
    if net:
        d.net = 1
        d.policy = 0
        if lights is not None:
            lv = [np.asarray(l, dtype=np.float64).reshape(-1, 6) for l in lights]
            if len(lv) != len(rect_list):
                raise ValueError("one light array per map")
            loff = np.zeros(len(lv) + 1, dtype=np.int32)
            for i, l in enumerate(lv):
                loff[i + 1] = loff[i] + len(l)
            lights_a = np.ascontiguousarray(np.concatenate(lv) if lv else np.zeros((0, 6)))
            size_a = np.ascontiguousarray(np.tile(np.asarray(map_size, np.float64), (len(lv), 1)))
            d.lights = lights_a.ctypes.data_as(_F64P)
            d.map_light_off = loff.ctypes.data_as(_I32P)
            d.map_size = size_a.ctypes.data_as(_F64P)
            keep += [lights_a, loff, size_a]
    return d, keep


_DEFAULTS = dict(max_slots=0, obs_ring=0, chunk_steps=32, policy=True, lanes=0, warps=0, ctas=0,
                 substeps=2, iterations=4, h=1 / 120, lin_drag=3.0, ang_drag=3.0, max_speed=360.0,
                 max_ang_speed=18.0, grip_slip_max=150.0, grip_cooldown=0.05, net=False, lights=None,
                 map_size=(1440.0, 810.0), slice_ms=0.0)


def plan(maps, hbm_budget, **kw):
    """(slots, bytes per slot) the server would have: pure host arithmetic."""
    o = dict(_DEFAULTS, **kw)
    d, keep = _desc(maps, hbm_budget, **o)
    cap, ps = C.c_int32(), C.c_uint64()
    _check(_lib().kr_server_plan(C.byref(d), C.byref(cap), C.byref(ps)), None)
    return cap.value, ps.value


def policy_eps(seed, pair, n):
    """The device's eps(seed, pair, 0..n) (standard normal numbers)."""
    out = np.zeros(n, dtype=np.float32)
    _check(_lib().kr_policy_eps(seed, pair, n, out.ctypes.data_as(_F32P)), None)
    return out


class Server:
    """One rollout server handle (kr_server).  Keywords as kr_server_desc:
    max_slots, chunk_steps, obs_ring, policy, net, lights, ... and slice_ms
    (> 0: one partition in preemptible time slices of that many ms, requests
    completing while their slice runs; 0: two partitions in rounds of
    chunk_steps env steps)."""

    def __init__(self, maps, hbm_budget, **kw):
        o = dict(_DEFAULTS, **kw)
        d, keep = _desc(maps, hbm_budget, **o)
        self.h = C.c_void_p()
        _check(_lib().kr_server_create(C.byref(d), C.byref(self.h)), None)

    def close(self):
        if getattr(self, "h", None) and self.h.value:
            _lib().kr_server_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def now(self) -> float:
        return _lib().kr_server_now(self.h)

    def submit(self, population, horizon, arms, segs, map_id, x=0.0, y=0.0, angle=0.0, theta=None,
               sigma=0.0, seed=0, tone=0.5, arrival=-1.0, xs=None, ys=None, angles=None,
               control_seeds=None, first_individual=0) -> int:
        """Queue a request; x, y, angle is the common spawn pose, or xs, ys,
        angles one pose per individual; control_seeds (no theta) one control
        stream seed per individual; first_individual (even): the index of
        this request's first individual when a population is split over
        several servers (its pairs' eps and streams are then the whole
        population's)."""
        th = None if theta is None else np.ascontiguousarray(theta, dtype=np.float32).ravel()
        per = None
        if xs is not None:
            per = [np.ascontiguousarray(v, dtype=np.float64) for v in (xs, ys, angles)]
        cs = None if control_seeds is None else np.ascontiguousarray(control_seeds, dtype=np.uint32)
        ptrs = tuple(v.ctypes.data_as(_F64P) for v in per) if per else (None, None, None)
        r = Request(int(population), int(horizon), int(arms), int(segs), int(map_id), float(x),
                    float(y), float(angle), *ptrs,
                    cs.ctypes.data_as(C.POINTER(C.c_uint32)) if cs is not None else None,
                    float(tone),
                    th.ctypes.data_as(_F32P) if th is not None else None,
                    0 if th is None else th.size, float(sigma), int(seed) & (2**64 - 1),
                    float(arrival), int(first_individual))
        rid = C.c_int64()
        _check(_lib().kr_server_submit(self.h, C.byref(r), C.byref(rid)), self.h)
        return rid.value

    def submit_many(self, horizon, arms, segs, map_id, xs, ys, angles, control_seeds=None,
                    tone=0.5, arrival=-1.0):
        """One single-creature request per row (its pose, control stream
        seed and horizon), queued with one C call; returns the ids."""
        n = len(horizon)
        a = np.zeros(n, dtype=REQUEST_DTYPE)
        keep = [np.ascontiguousarray(v, dtype=np.float64) for v in (xs, ys, angles)]
        a["population"] = 1
        a["horizon"] = horizon
        a["arms"] = arms
        a["segs"] = segs
        a["map_id"] = map_id
        for f, v in zip(("xs", "ys", "angles"), keep):
            a[f] = v.ctypes.data + 8 * np.arange(n, dtype=np.uint64)
        if control_seeds is not None:
            cs = np.ascontiguousarray(control_seeds, dtype=np.uint32)
            keep.append(cs)
            a["control_seeds"] = cs.ctypes.data + 4 * np.arange(n, dtype=np.uint64)
        a["tone"] = tone
        a["arrival"] = arrival
        ids = np.zeros(n, dtype=np.int64)
        done = C.c_int32()
        _check(_lib().kr_server_submit_batch(self.h, a.ctypes.data, n, ids.ctypes.data_as(_I64P),
                                             C.byref(done)), self.h)
        return ids

    def results_many(self, ids, populations=None, release=False):
        """Results of completed requests, concatenated in id order
        (sum of populations, RESULT_WORDS), and their times (len(ids), 3)."""
        ids = np.ascontiguousarray(ids, dtype=np.int64)
        total = len(ids) if populations is None else int(np.sum(populations))
        out = np.zeros((total, RESULT_WORDS), dtype=np.float64)
        t = np.zeros((len(ids), 3), dtype=np.float64)
        _check(_lib().kr_server_result_batch(self.h, ids.ctypes.data_as(_I64P), len(ids),
                                             out.ctypes.data_as(_F64P), t.ctypes.data_as(_F64P),
                                             1 if release else 0), self.h)
        return out, t

    def pump(self) -> bool:
        busy = C.c_int32()
        _check(_lib().kr_server_pump(self.h, C.byref(busy)), self.h)
        return bool(busy.value)

    def drain(self):
        _check(_lib().kr_server_drain(self.h), self.h)

    def poll(self, cap=4096):
        ids = np.zeros(cap, dtype=np.int64)
        n = C.c_int32()
        _check(_lib().kr_server_poll(self.h, ids.ctypes.data_as(_I64P), cap, C.byref(n)), self.h)
        return [int(i) for i in ids[: n.value]]

    def result(self, rid, population):
        out = np.zeros((population, RESULT_WORDS), dtype=np.float64)
        t = np.zeros(3, dtype=np.float64)
        _check(_lib().kr_server_result(self.h, rid, out.ctypes.data_as(_F64P),
                                       t.ctypes.data_as(_F64P)), self.h)
        return {"results": out, "arrival": t[0], "admitted": t[1], "completed": t[2]}

    def release(self, rid):
        _check(_lib().kr_server_release(self.h, rid), self.h)

    def stats(self):
        s = Stats()
        _check(_lib().kr_server_get_stats(self.h, C.byref(s)), self.h)
        return {f: getattr(s, f) for f, _ in Stats._fields_}
