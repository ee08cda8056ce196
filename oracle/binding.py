"""ctypes binding of the CPU oracle -- TEST INFRASTRUCTURE ONLY.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's ``cpu_baseline`` leg
import this module.  It wraps ``oracle/liboracle.so`` (built by
``oracle/Makefile``), the C restatement of src/physics/xpbd.js (ref64) and
tools/f32solver.mjs (ref32) together with the world builders of
src/world/map.js, src/body/kraken.js and src/sim/core.js.

The wrappers mirror the reference's JS objects closely enough that a test
reads like tools/harness.js: ``World`` ~ XpbdWorld, ``Sim`` ~ createSim's
return value, ``Kraken`` ~ the object spawnKraken returns.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
OPCOUNT_PATH = os.path.join(HERE, "liboracle_opcount.so")

C_PIN, C_ANGLE, C_GRIP = 0, 1, 2
MAX_ARMS = 16
MAX_SEGS = 16

FIELDS = ["type", "a", "b", "lax", "lay", "lbx", "lby", "compliance", "lambda",
          "lambdaX", "lambdaY", "broken", "breakForce", "force", "target", "rest",
          "minAngle", "maxAngle", "owner", "color"]
FIELD_ID = {n: i for i, n in enumerate(FIELDS)}
ARRAYS = ["px", "py", "ppx", "ppy", "vx", "vy", "ang", "angP", "av", "im", "ii",
          "fx", "fy", "tq"]
ARRAY_ID = {n: i for i, n in enumerate(ARRAYS)}


class KrakenStruct(C.Structure):
    _fields_ = [
        ("mantle", C.c_int), ("nArms", C.c_int), ("nSegs", C.c_int),
        ("segs", (C.c_int * MAX_SEGS) * MAX_ARMS),
        ("motors", (C.c_int * MAX_SEGS) * MAX_ARMS),
        ("grip", C.c_int * MAX_ARMS),
        ("tip", C.c_int * MAX_ARMS),
        ("relAng", C.c_double * MAX_ARMS),
        ("spawnX", C.c_double), ("spawnY", C.c_double), ("spawnAngle", C.c_double),
    ]


def build() -> None:
    """Compile the oracle with its Makefile (gcc, -ffp-contract=off)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


_LIBS: dict[str, C.CDLL] = {}


def lib(opcount: bool = False) -> C.CDLL:
    path = OPCOUNT_PATH if opcount else LIB_PATH
    if path in _LIBS:
        return _LIBS[path]
    if not os.path.exists(path):
        build()
    L = C.CDLL(path)
    d, i, u32, vp = C.c_double, C.c_int, C.c_uint32, C.c_void_p
    dp, ip, u32p = C.POINTER(C.c_double), C.POINTER(C.c_int), C.POINTER(C.c_uint32)
    sig = {
        "or_mulberry32_next": (u32, [u32p, dp]),
        "or_rnd": (d, [u32p]),
        "or_make_map": (i, [d, d, d, i, i, d, u32, dp, i]),
        "or_sdf": (i, [dp, i, d, d, dp, dp, dp]),
        "or_find_spawn": (None, [dp, i, d, d, d, u32p, dp, dp]),
        "or_world_new": (vp, [i, i, d, d, d, d, d]),
        "or_world_free": (None, [vp]),
        "or_world_n": (i, [vp]), "or_world_nc": (i, [vp]), "or_world_np": (i, [vp]),
        "or_world_array": (dp, [vp, i]),
        "or_add_body": (i, [vp, d, d, d, d, d]),
        "or_add_collision_point": (None, [vp, i, d, d, d]),
        "or_get_collision_point": (None, [vp, i, ip, dp, dp, dp]),
        "or_add_constraint": (i, [vp, i, i, i, d, d, d, d, d]),
        "or_con_get": (d, [vp, i, i]),
        "or_con_set": (None, [vp, i, i, d]),
        "or_world_list": (i, [vp, i]),
        "or_world_set_list": (None, [vp, ip, i]),
        "or_world_set_rects": (None, [vp, dp, i]),
        "or_world_color_info": (None, [vp, u32p, u32p]),
        "or_world_stats": (None, [vp, dp, dp, ip, C.POINTER(C.c_long), ip]),
        "or_assign_color": (i, [u32p, i, i]),
        "or_ensure_colored": (None, [vp]),
        "or_group_by_color": (None, [vp]),
        "or_step": (None, [vp]), "or_substep": (None, [vp]),
        "or_solve_collisions": (None, [vp]),
        "or_f32ify": (None, [vp]), "or_f32_round_state": (None, [vp]),
        "or_step32": (None, [vp]),
        "or_f32_op_count": (C.c_uint64, []), "or_f32_op_count_reset": (None, []),
        "or_spawn_kraken": (i, [vp, d, d, d, i, i, d, C.POINTER(KrakenStruct)]),
        "or_tip_position": (None, [vp, C.POINTER(KrakenStruct), i, dp, dp]),
        "or_attach_grip": (None, [vp, C.POINTER(KrakenStruct), i, d]),
        "or_release_grip": (None, [vp, C.POINTER(KrakenStruct), i]),
        "or_tone_to_compliance": (d, [d]),
        "or_adhesion_to_break_force": (d, [d]),
        "or_arm_reach": (d, [i]),
        "or_sim_create": (vp, [u32, i, d, d, i, i, d, i, i]),
        "or_sim_free": (None, [vp]),
        "or_sim_new": (vp, [d, d, dp, i, i, i, d]),
        "or_sim_add_creature": (i, [vp, d, d, d, i, i]),
        "or_sim_world": (vp, [vp]),
        "or_sim_rects": (i, [vp, dp, i]),
        "or_sim_ncreatures": (i, [vp]),
        "or_sim_kraken": (None, [vp, i, C.POINTER(KrakenStruct)]),
        "or_sim_set_reflex": (None, [vp, d, d]),
        "or_apply_control": (None, [vp, i, d, dp, dp, dp]),
        "or_apply_control_motors": (None, [vp, i, d, dp, dp]),
        "or_sim_reflex_state": (None, [vp, i, dp, dp]),
        "or_read_proprio": (i, [vp, i, dp]),
        "or_sim_step": (None, [vp]), "or_sim_step32": (None, [vp]),
        "or_measure_reach": (d, [dp, i, d, d, d]),
        "or_sim_set_spawn_reach": (None, [vp, i, d]),
        "or_sim_pre_step": (None, [vp]), "or_sim_post_step": (None, [vp]),
        "or_sim_metrics": (None, [vp, i, C.POINTER(Metrics)]),
        "or_bench_rollouts": (i, [i, dp, ip, ip, ip, ip, dp, dp, dp, u32p, ip, d, i, i, i, d, d, d, i, d, i,
                                  C.POINTER(C.c_longlong), dp, dp]),
        "or_score": (d, [C.POINTER(Metrics)]),
        "or_net_new": (vp, [vp, dp, i]),
        "or_net_free": (None, [vp]),
        "or_net_param_count": (i, [i]),
        "or_net_forward": (None, [C.POINTER(C.c_float), C.POINTER(C.c_float), C.POINTER(C.c_float),
                                  C.POINTER(C.c_float), i, i]),
        "or_net_step": (i, [vp, C.POINTER(C.c_float), i, ip, i]),
        "or_net_io": (None, [vp, i, C.POINTER(C.c_float), C.POINTER(C.c_float)]),
        "or_net_echo": (None, [vp, i, ip, ip]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _LIBS[path] = L
    return L


def _dp(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


# --------------------------------------------------------------------------
# map.js
# --------------------------------------------------------------------------
class Rng:
    """mulberry32 (map.js:11-20)."""

    def __init__(self, seed: int):
        self.state = C.c_uint32(seed & 0xFFFFFFFF)

    def __call__(self) -> float:
        return lib().or_rnd(C.byref(self.state))


def make_map_rects(width=1440.0, height=810.0, seed=1, density=0.48, wall=14.0,
                   cols=4, rows=3) -> np.ndarray:
    """makeMap rect list (map.js:22-59) as an (n, 4) float64 array x, y, w, h."""
    buf = np.zeros((512, 4))
    n = lib().or_make_map(width, height, wall, cols, rows, density, seed & 0xFFFFFFFF,
                          _dp(buf), 512)
    return buf[:n].copy()


def sdf(rects: np.ndarray, x: float, y: float):
    """makeSdf (map.js:91-118): (d, nx, ny) or None."""
    r = np.ascontiguousarray(rects, dtype=np.float64)
    d, nx, ny = C.c_double(), C.c_double(), C.c_double()
    ok = lib().or_sdf(_dp(r), len(r), x, y, C.byref(d), C.byref(nx), C.byref(ny))
    return (d.value, nx.value, ny.value) if ok else None


def find_spawn(rects, width, height, clearance, rng: Rng):
    r = np.ascontiguousarray(rects, dtype=np.float64)
    x, y = C.c_double(), C.c_double()
    lib().or_find_spawn(_dp(r), len(r), width, height, clearance, C.byref(rng.state),
                        C.byref(x), C.byref(y))
    return x.value, y.value


def tone_to_compliance(t: float) -> float:
    return lib().or_tone_to_compliance(t)


def adhesion_to_break_force(a: float) -> float:
    return lib().or_adhesion_to_break_force(a)


def arm_reach(segs: int = 7) -> float:
    return lib().or_arm_reach(segs)


# --------------------------------------------------------------------------
# XpbdWorld
# --------------------------------------------------------------------------
class Constraint:
    """Live view of one constraint (JS object identity = creation id)."""

    __slots__ = ("_w", "id")

    def __init__(self, world: "World", cid: int):
        object.__setattr__(self, "_w", world)
        object.__setattr__(self, "id", cid)

    def __getattr__(self, name):
        if name in FIELD_ID:
            v = self._w.L.or_con_get(self._w.ptr, self.id, FIELD_ID[name])
            if name in ("type", "a", "b", "owner", "color"):
                return int(v)
            if name == "broken":
                return bool(v)
            return v
        raise AttributeError(name)

    def __setattr__(self, name, value):
        if name not in FIELD_ID:
            raise AttributeError(name)
        self._w.L.or_con_set(self._w.ptr, self.id, FIELD_ID[name], float(value))


class World:
    """XpbdWorld restatement (xpbd.js:188-505); owns the C world unless borrowed."""

    def __init__(self, substeps=2, iterations=4, h=1 / 120, linDrag=3.0, angDrag=3.0,
                 maxSpeed=360.0, maxAngSpeed=18.0, _ptr=None, _owner=None,
                 opcount=False):
        self.L = lib(opcount)
        if _ptr is None:
            self.ptr = self.L.or_world_new(substeps, iterations, h, linDrag, angDrag,
                                           maxSpeed, maxAngSpeed)
            self._own = True
        else:
            self.ptr = _ptr
            self._own = False
        self._owner = _owner
        self.substeps, self.iterations, self.h = substeps, iterations, h

    def __del__(self):
        if getattr(self, "_own", False) and self.ptr:
            self.L.or_world_free(self.ptr)
            self.ptr = None

    # -- sizes and arrays --
    @property
    def n(self) -> int:
        return self.L.or_world_n(self.ptr)

    @property
    def nC(self) -> int:
        return self.L.or_world_nc(self.ptr)

    @property
    def nP(self) -> int:
        return self.L.or_world_np(self.ptr)

    def arr(self, name: str) -> np.ndarray:
        """Live numpy view of one body array (valid until the next add_body)."""
        p = self.L.or_world_array(self.ptr, ARRAY_ID[name])
        return np.ctypeslib.as_array(p, shape=(self.n,))

    def __getattr__(self, name):
        if name in ARRAY_ID:
            return self.arr(name)
        raise AttributeError(name)

    # -- building --
    def add_body(self, x, y, angle, mass, inertia) -> int:
        return self.L.or_add_body(self.ptr, x, y, angle, mass, inertia)

    def add_collision_point(self, body, lx, ly, r):
        self.L.or_add_collision_point(self.ptr, body, lx, ly, r)

    def coll_pts(self):
        out = []
        b, lx, ly, r = C.c_int(), C.c_double(), C.c_double(), C.c_double()
        for i in range(self.nP):
            self.L.or_get_collision_point(self.ptr, i, C.byref(b), C.byref(lx),
                                          C.byref(ly), C.byref(r))
            out.append((b.value, lx.value, ly.value, r.value))
        return out

    def add_constraint(self, type_, a, b, lax, lay, lbx, lby, compliance=0.0) -> Constraint:
        cid = self.L.or_add_constraint(self.ptr, type_, a, b, lax, lay, lbx, lby, compliance)
        return Constraint(self, cid)

    def con(self, cid: int) -> Constraint:
        return Constraint(self, cid)

    @property
    def constraints(self):
        """Solve order (XpbdWorld.constraints) as Constraint views."""
        return [Constraint(self, self.L.or_world_list(self.ptr, k)) for k in range(self.nC)]

    def list_ids(self) -> np.ndarray:
        return np.array([self.L.or_world_list(self.ptr, k) for k in range(self.nC)],
                        dtype=np.int32)

    def set_list(self, ids):
        a = np.ascontiguousarray(ids, dtype=np.int32)
        self.L.or_world_set_list(self.ptr, a.ctypes.data_as(C.POINTER(C.c_int)), len(a))

    def set_rects(self, rects):
        r = np.ascontiguousarray(rects, dtype=np.float64).reshape(-1, 4)
        self.L.or_world_set_rects(self.ptr, _dp(r), len(r))

    def color_info(self):
        off = (C.c_uint32 * 16)()
        cnt = (C.c_uint32 * 16)()
        self.L.or_world_color_info(self.ptr, off, cnt)
        return list(off), list(cnt)

    def ensure_colored(self):
        self.L.or_ensure_colored(self.ptr)

    def group_by_color(self):
        self.L.or_group_by_color(self.ptr)

    # -- physics --
    def step(self):
        self.L.or_step(self.ptr)

    def solve_collisions(self):
        self.L.or_solve_collisions(self.ptr)

    def f32ify(self):
        self.L.or_f32ify(self.ptr)

    def round_state(self):
        self.L.or_f32_round_state(self.ptr)

    def step32(self):
        self.L.or_step32(self.ptr)

    @property
    def stats(self):
        ms, ma, nan, col, br = C.c_double(), C.c_double(), C.c_int(), C.c_long(), C.c_int()
        self.L.or_world_stats(self.ptr, C.byref(ms), C.byref(ma), C.byref(nan),
                              C.byref(col), C.byref(br))
        return {"maxSpeed": ms.value, "maxAngSpeed": ma.value, "nan": nan.value,
                "collisions": col.value, "broken": br.value}

    # -- kraken.js --
    def spawn_kraken(self, x, y, angle, arms=6, segs=7, curl=0.28) -> "Kraken":
        k = KrakenStruct()
        rc = self.L.or_spawn_kraken(self.ptr, x, y, angle, arms, segs, curl, C.byref(k))
        if rc < 0:
            raise ValueError("bad body shape")
        return Kraken(self, k)


class Kraken:
    """The object spawnKraken returns (kraken.js:64-148)."""

    def __init__(self, world: World, k: KrakenStruct):
        self.world = world
        self.s = k
        self.mantle = k.mantle
        self.n_arms, self.n_segs = k.nArms, k.nSegs
        self.segs = [[k.segs[a][i] for i in range(k.nSegs)] for a in range(k.nArms)]
        self.motors = [[k.motors[a][i] for i in range(k.nSegs)] for a in range(k.nArms)]
        self.grips = [k.grip[a] for a in range(k.nArms)]
        self.tips = [k.tip[a] for a in range(k.nArms)]
        self.spawn = (k.spawnX, k.spawnY, k.spawnAngle)

    def tip_position(self, arm):
        x, y = C.c_double(), C.c_double()
        self.world.L.or_tip_position(self.world.ptr, C.byref(self.s), arm, C.byref(x), C.byref(y))
        return x.value, y.value

    def attach_grip(self, arm, break_force):
        self.world.L.or_attach_grip(self.world.ptr, C.byref(self.s), arm, break_force)

    def release_grip(self, arm):
        self.world.L.or_release_grip(self.world.ptr, C.byref(self.s), arm)

    def grip(self, arm) -> Constraint:
        return self.world.con(self.grips[arm])


METRIC_FIELDS = ("score", "steps", "pathLen", "maxDisplacement", "spawnReach", "angularAccum",
                 "forwardProg", "gripPullProg", "anchoredSteps", "freeMove", "energySpent",
                 "gripCycles", "strides", "attachEvents", "x", "y")


class Metrics(C.Structure):
    """or_metrics: postStep's accumulators (core.js:297-356) and score."""
    _fields_ = [(f, C.c_double) for f in METRIC_FIELDS] + [("spawnDistMax", C.c_double)]


def measure_reach(rects, reach, x, y) -> float:
    """measureReach (fitness.js:74-88) over rects x y w h, rays up to 3.5 reach."""
    r = np.ascontiguousarray(rects, dtype=np.float64).reshape(-1, 4)
    return lib().or_measure_reach(_dp(r), len(r), reach, x, y)


class Sim:
    """createSim (core.js:37-74) with prey 0; physics, colouring and reflex only.

    With ``rects`` given, an empty sim on that map instead; creatures are then
    added at explicit poses with :meth:`add_creature`."""

    def __init__(self, seed=1, creatures=1, width=1440.0, height=810.0, substeps=2,
                 iterations=4, h=1 / 120, arms=6, segs=7, opcount=False, rects=None):
        self.L = lib(opcount)
        if rects is None:
            self.ptr = self.L.or_sim_create(seed & 0xFFFFFFFF, creatures, width, height,
                                            substeps, iterations, h, arms, segs)
        else:
            r = np.ascontiguousarray(rects, dtype=np.float64).reshape(-1, 4)
            self.ptr = self.L.or_sim_new(width, height, _dp(r), len(r), substeps, iterations, h)
        self.world = World(substeps, iterations, h, _ptr=self.L.or_sim_world(self.ptr),
                           _owner=self, opcount=opcount)
        buf = np.zeros((512, 4))
        n = self.L.or_sim_rects(self.ptr, _dp(buf), 512)
        self.rects = buf[:n].copy()
        self.width, self.height = width, height
        self.creatures = []
        for i in range(self.L.or_sim_ncreatures(self.ptr)):
            k = KrakenStruct()
            self.L.or_sim_kraken(self.ptr, i, C.byref(k))
            self.creatures.append(Kraken(self.world, k))

    def __del__(self):
        if getattr(self, "ptr", None):
            self.L.or_sim_free(self.ptr)
            self.ptr = None

    def add_creature(self, x, y, angle, arms=6, segs=7) -> "Kraken":
        i = self.L.or_sim_add_creature(self.ptr, x, y, angle, arms, segs)
        if i < 0:
            raise ValueError("bad body shape")
        k = KrakenStruct()
        self.L.or_sim_kraken(self.ptr, i, C.byref(k))
        kr = Kraken(self.world, k)
        self.creatures.append(kr)
        return kr

    def set_reflex(self, slip_max=150.0, cooldown=0.05):
        self.L.or_sim_set_reflex(self.ptr, slip_max, cooldown)

    def apply_control(self, ci, tone, shoulder, curl, adhesion):
        s = np.ascontiguousarray(shoulder, dtype=np.float64)
        c = np.ascontiguousarray(curl, dtype=np.float64)
        a = np.ascontiguousarray(adhesion, dtype=np.float64)
        self.L.or_apply_control(self.ptr, ci, tone, _dp(s), _dp(c), _dp(a))

    def apply_control_motors(self, ci, tone, targets, adhesion):
        t = np.ascontiguousarray(targets, dtype=np.float64)
        a = np.ascontiguousarray(adhesion, dtype=np.float64)
        self.L.or_apply_control_motors(self.ptr, ci, tone, _dp(t), _dp(a))

    def reflex_state(self, ci):
        A = self.creatures[ci].n_arms
        cd = np.zeros(A)
        ad = np.zeros(A)
        self.L.or_sim_reflex_state(self.ptr, ci, _dp(cd), _dp(ad))
        return cd, ad

    def read_proprio(self, ci) -> np.ndarray:
        out = np.zeros(6 * MAX_ARMS + 6)
        n = self.L.or_read_proprio(self.ptr, ci, _dp(out))
        return out[:n].copy()

    def step(self):
        self.L.or_sim_step(self.ptr)

    def step32(self):
        self.L.or_sim_step32(self.ptr)

    def pre_step(self):
        """preStep of every creature (core.js:291-294)."""
        self.L.or_sim_pre_step(self.ptr)

    def post_step(self):
        """postStep of every creature (core.js:297-356)."""
        self.L.or_sim_post_step(self.ptr)

    def set_spawn_reach(self, ci, reach):
        self.L.or_sim_set_spawn_reach(self.ptr, ci, reach)

    def metrics(self, ci) -> dict:
        """postStep accumulators and score (fitness.js:115-172) of creature ci."""
        m = Metrics()
        self.L.or_sim_metrics(self.ptr, ci, C.byref(m))
        return {f: getattr(m, f) for f in METRIC_FIELDS}


def _fp(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def net_param_count(arms: int) -> int:
    """net.js weightCount for an arms-armed body (n_in = 10 arms + 45)."""
    return lib().or_net_param_count(arms)


def net_forward(w, x, n_out):
    """forwardInto (net.js:71-98) of one genome on one input vector."""
    w = np.ascontiguousarray(w, dtype=np.float32)
    x = np.ascontiguousarray(x, dtype=np.float32)
    out = np.zeros(n_out, np.float32)
    scratch = np.zeros(48, np.float32)
    lib().or_net_forward(_fp(w), _fp(x), _fp(out), _fp(scratch), len(x), n_out)
    return out


class NetSim:
    """The trainer's controller over a :class:`Sim`'s creatures: senses
    without entities, the recurrent net and trainStep (train.js:233-249).
    ``lights`` are the map's lights, rows x y r ir ph sp."""

    def __init__(self, sim: Sim, lights=None):
        self.sim = sim
        self.L = sim.L
        lv = np.ascontiguousarray(np.zeros((0, 6)) if lights is None else lights, dtype=np.float64)
        self.ptr = self.L.or_net_new(sim.ptr, _dp(lv), len(lv))
        if not self.ptr:
            raise ValueError("too many lights")

    def __del__(self):
        if getattr(self, "ptr", None):
            self.L.or_net_free(self.ptr)
            self.ptr = None

    def step(self, genomes, individual, f32=True):
        g = np.ascontiguousarray(genomes, dtype=np.float32)
        ind = np.ascontiguousarray(individual, dtype=np.int32)
        rc = self.L.or_net_step(self.ptr, _fp(g), g.shape[-1], ind.ctypes.data_as(C.POINTER(C.c_int)),
                                1 if f32 else 0)
        if rc != 0:
            raise ValueError("genome size does not match a creature's arm count")

    def io(self, ci):
        A = self.sim.creatures[ci].n_arms
        x = np.zeros(10 * A + 45, np.float32)
        out = np.zeros(3 * A + 2, np.float32)
        self.L.or_net_io(self.ptr, ci, _fp(x), _fp(out))
        return x, out

    def echo(self, ci):
        e, p = C.c_int(), C.c_int()
        self.L.or_net_echo(self.ptr, ci, C.byref(e), C.byref(p))
        return e.value, p.value


def bench_rollouts(maps, map_id, arms, segs, x, y, angle, seed, horizon, threads, limit_s=0.0,
                   tone=0.5, period=6, substeps=2, iterations=4, h=1 / 120, width=1440.0, height=810.0,
                   metrics=False, f32=False):
    """The timed CPU baseline (xpbd_bench.c): every creature in its own
    one-creature world, driven per env step by its mulberry32 control stream,
    applyControl, preStep, the FP64 step and postStep, on `threads` POSIX
    threads over contiguous creature ranges, with no Python in the loop.
    Returns (creature-steps done, seconds) and, with metrics, each creature's
    final mantle x, y, path length and score (n, 4); f32: the f32 emulation's
    step instead of the FP64 one (for checks)."""
    L = lib()
    rects = np.ascontiguousarray(np.concatenate([np.asarray(m, np.float64).reshape(-1, 4) for m in maps]))
    off = np.zeros(len(maps) + 1, np.int32)
    off[1:] = np.cumsum([len(np.asarray(m).reshape(-1, 4)) for m in maps])
    ii = [np.ascontiguousarray(a, dtype=np.int32) for a in (map_id, arms, segs, horizon)]
    dd = [np.ascontiguousarray(a, dtype=np.float64) for a in (x, y, angle)]
    sd = np.ascontiguousarray(seed, dtype=np.uint32)
    n = len(sd)
    out = np.zeros((n, 4)) if metrics else None
    steps, el = C.c_longlong(), C.c_double()
    ipp = C.POINTER(C.c_int)
    rc = L.or_bench_rollouts(n, _dp(rects), off.ctypes.data_as(ipp), ii[0].ctypes.data_as(ipp),
                             ii[1].ctypes.data_as(ipp), ii[2].ctypes.data_as(ipp), _dp(dd[0]), _dp(dd[1]),
                             _dp(dd[2]), sd.ctypes.data_as(C.POINTER(C.c_uint32)), ii[3].ctypes.data_as(ipp),
                             tone, period, substeps, iterations, h, width, height, threads, limit_s,
                             1 if f32 else 0, C.byref(steps), C.byref(el), _dp(out) if metrics else None)
    if rc != 0:
        raise RuntimeError(f"or_bench_rollouts: status {rc}")
    return (steps.value, el.value, out) if metrics else (steps.value, el.value)
