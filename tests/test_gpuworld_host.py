"""Host-only parts of the gpuworld drop-in: field offsets of mirrorInto and
packControls (harness.js:895-971), collision-point grouping, and the C ABI
exports (library loads, every declared symbol present -- no device calls)."""
import ctypes
import math
import os
import re

import numpy as np
import pytest

from kraken_3_gpu_b200 import _native, core, gpuworld

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_mirror_fields():
    # harness G8a, harness.js:895-942
    sim = core.create_sim(seed=31, creatures=2)
    w = sim["world"]
    nB, nC = w.n, len(w.constraints)
    bd = np.zeros(nB * gpuworld.GPU_STRIDES["body"], dtype=np.float32)
    cd = np.zeros(nC * gpuworld.GPU_STRIDES["constraint"], dtype=np.float32)
    cu = cd.view(np.uint32)
    for i in range(nB):
        o = i * 12
        bd[o] = 100 + i * 0.5
        bd[o + 1] = -200 + i * 0.25
        bd[o + 4] = 1 + i * 0.01
        bd[o + 5] = -2 - i * 0.01
        bd[o + 6] = 0.3 + i * 0.001
        bd[o + 8] = 0.05 + i * 0.002
    for k in range(nC):
        o = k * 20
        cd[o + 13] = 0.5 + k * 0.001
        cd[o + 14] = -0.25 + k * 0.001
        cd[o + 15] = k * 0.002
        cu[o + 17] = k % 2
    stats = gpuworld.mirrorInto(w, bd, cd)
    for i in range(nB):
        assert w.px[i] == bd[i * 12] and w.py[i] == bd[i * 12 + 1]
        assert w.vx[i] == bd[i * 12 + 4] and w.vy[i] == bd[i * 12 + 5]
        assert w.ang[i] == bd[i * 12 + 6] and w.av[i] == bd[i * 12 + 8]
    inv_h = 1 / w.h
    n_grips = 0
    for k, c in enumerate(w.constraints):
        assert c.lambda_ == cd[k * 20 + 15]
        assert c.broken == (k % 2 == 1)
        if c.type == 2:
            n_grips += 1
            fx, fy = float(cd[k * 20 + 13]), float(cd[k * 20 + 14])
            assert c.lambdaX == fx and c.lambdaY == fy
            assert c.force == math.hypot(fx, fy) * inv_h
    exp_max_v = max(math.sqrt(float(bd[i * 12 + 4]) ** 2 + float(bd[i * 12 + 5]) ** 2)
                    for i in range(nB))
    assert stats["maxSpeed"] == exp_max_v and stats["nan"] == 0
    assert nB == 86 and nC == 180 and n_grips == 12


def test_pack_controls():
    # harness G8b, harness.js:944-971
    sim = core.create_sim(seed=33, creatures=1)
    w = sim["world"]
    nC = len(w.constraints)
    cd = np.zeros(nC * 20, dtype=np.float32)
    cu = cd.view(np.uint32)
    for k, c in enumerate(w.constraints):
        c.compliance = 0.123 + k * 1e-4
        c.target = 0.01 * k
        c.breakForce = math.inf if k % 3 == 0 else 5 + k
        c.broken = k % 2 == 0
        c.lbx = 11 + k
        c.lby = -22 - k
    gpuworld.packControls(w, cd)
    f32 = np.float32
    for k, c in enumerate(w.constraints):
        o = k * 20
        assert cd[o + 6] == f32(c.lbx) and cd[o + 7] == f32(c.lby)
        assert cd[o + 8] == f32(c.compliance) and cd[o + 10] == f32(c.target)
        assert cd[o + 16] == f32(min(c.breakForce, 1e30))
        assert cu[o + 17] == (1 if c.broken else 0)


def test_group_coll_points_stable():
    sim = core.create_sim(seed=5, creatures=2)
    w = sim["world"]
    g = gpuworld.groupCollPoints(w.collPts, w.n)
    order, rng = g["order"], g["range"]
    for b in range(w.n):
        pts = [w.collPts[int(order[rng[b] + q])] for q in range(rng[w.n + b])]
        assert all(p.body == b for p in pts)
        idx = [int(order[rng[b] + q]) for q in range(rng[w.n + b])]
        assert idx == sorted(idx)
    with pytest.raises(ValueError):
        gpuworld.groupCollPoints(w.collPts, 3)


def _declared_symbols():
    syms = set()
    inc = os.path.join(ROOT, "include")
    for f in os.listdir(inc):
        if f.endswith(".h"):
            src = open(os.path.join(inc, f)).read()
            syms |= set(re.findall(r"\b(kr_[a-z0-9_]+)\s*\(", src))
    return syms


def test_c_abi_exports_every_declared_symbol():
    lib = _native.lib()
    syms = _declared_symbols()
    assert "kr_create" in syms and "kr_step" in syms
    for s in sorted(syms):
        assert hasattr(lib, s), f"{s} declared in include/ but not exported"


def test_create_rejects_implausible_params_without_device():
    # writeStatic guards (gpuworld.js:224-229) fire before any device call
    from kraken_3_gpu_b200 import xpbd
    sim = core.create_sim(seed=1, creatures=1)
    w = sim["world"]
    w.iterations = 0
    with pytest.raises(_native.KrError) as e:
        gpuworld.create(w, sim["map"])
    assert e.value.code == _native.KR_ERR_INVALID and "iterations" in str(e.value)
    w.iterations = 4
    w.h = 1.5
    with pytest.raises(_native.KrError):
        gpuworld.create(w, sim["map"])
    empty = {"rects": [], "width": 1440, "height": 810}
    w.h = 1 / 120
    with pytest.raises(_native.KrError) as e:
        gpuworld.create(w, empty)
    assert "nRects" in str(e.value)


def test_no_alloc_step_rejects_misaligned_buffers_without_device():
    # kr_step_noalloc moves bodies, forces, constraints and collision points
    # as 16-byte vectors and reads rects / collRange as words: a pointer off
    # that alignment (a caller's pool may hand one out) is refused with
    # KR_ERR_INVALID before any CUDA call.  The addresses are never
    # dereferenced: the argument checks come first.
    L = _native.lib()
    L.kr_step_noalloc.restype = ctypes.c_int
    L.kr_step_noalloc.argtypes = [ctypes.POINTER(_native.SolverParams), ctypes.c_uint32, ctypes.c_uint32,
                                  ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                  ctypes.c_uint32, ctypes.c_void_p, ctypes.c_uint32, ctypes.c_void_p,
                                  ctypes.c_int32, ctypes.c_void_p]
    params = _native.SolverParams(1 / 120, 2, 4, 3.0, 3.0, 360.0, 18.0)
    base = 1 << 20
    ok = dict(bodies=base, cons=base + 4096, forces=base + 8192, rects=base + 12288,
              coll=base + 16384, rng=base + 20480)
    for name, off in (("bodies", 4), ("cons", 8), ("forces", 4), ("coll", 12), ("rects", 2), ("rng", 1)):
        a = dict(ok)
        a[name] += off
        rc = L.kr_step_noalloc(ctypes.byref(params), 43, 90, a["bodies"], a["cons"], a["forces"], a["rects"],
                               24, a["coll"], 92, a["rng"], 1, None)
        assert rc == _native.KR_ERR_INVALID, f"{name} + {off}: status {rc}"
