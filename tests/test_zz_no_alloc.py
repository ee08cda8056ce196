"""The allocation-free step entry point (kr_step_noalloc) against the
regular one (kr_create / kr_upload / kr_step).

Some callers cannot allocate GPU memory -- an application that owns every
device allocation through its own pool, or a latency-critical loop where a
cudaMalloc and its implicit synchronization are not allowed.  They call
kr_step_noalloc with their own device buffers; the library keeps its
scratch (the per-creature schedule) in one fixed-size device array.  This
test gives it the same world the regular entry point runs and checks that
two calls in a row produce the same bodies and constraints, bit for bit
(the tolerance of every other parity test here); it also runs 64 creatures
for ten steps per call straight against the f32 oracle, and checks that
worlds the kernel cannot take -- above the stated limits, an inconsistent
collRange (one whose counts wrap a 32-bit sum included), a bad body index,
a creature above the per-island capacity -- are rejected with the stated
code and leave the caller's buffers untouched.  It runs last so that a
failure here never hides another test's result.
"""
import ctypes as C

import numpy as np
import pytest

from kraken_3_gpu_b200 import _native, core, gpuworld
from kraken_3_gpu_b200.workloads import TONE, ControlStream
from oracle import binding as ob
from tests.scenarios import ulp_distance

pytestmark = pytest.mark.gpu

_F32P = C.POINTER(C.c_float)
_U32P = C.POINTER(C.c_uint32)


def _bind():
    L = _native.lib()
    L.kr_step_noalloc.restype = C.c_int
    L.kr_step_noalloc.argtypes = [C.POINTER(_native.SolverParams), C.c_uint32, C.c_uint32,
                                  C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32,
                                  C.c_void_p, C.c_uint32, C.c_void_p, C.c_int32, C.c_void_p]
    return L


def _world(seed=3, creatures=2, arms=6, segs=7, controls=None):
    sim = core.create_sim(seed=seed, creatures=creatures, arms=arms, segsPerArm=segs)
    w, m = sim["world"], sim["map"]
    g = gpuworld.create(w, m)
    gpuworld.upload(g)
    gpuworld.download(g)
    for ci, c in enumerate(sim["creatures"]):
        t, a = controls[ci] if controls else ControlStream(seed=40 + ci).at(0)
        core.apply_control_motors(c, TONE, t, a)
    gpuworld.uploadControls(g)
    rects = np.array([[r["x"], r["y"], r["w"], r["h"]] for r in m["rects"]], dtype=np.float32)
    grouped = gpuworld.groupCollPoints(w.collPts, w.n)
    coll = np.zeros((len(w.collPts), 4), dtype=np.float32)
    cu = coll.view(np.uint32)
    for o, idx in enumerate(grouped["order"]):
        p = w.collPts[int(idx)]
        cu[o, 0] = p.body
        coll[o, 1:] = (p.lx, p.ly, p.r)
    return w, g, rects, coll, np.ascontiguousarray(grouped["range"], dtype=np.uint32)


def test_no_alloc_step_matches_regular_step_twice():
    import torch

    L = _bind()
    w, g, rects, coll, rng = _world()
    nB, nC, nP, nR = w.n, len(w.constraints), len(w.collPts), len(rects)
    # the caller's own device buffers, filled with the state the regular
    # entry point holds right now
    dev = torch.device("cuda", 0)
    bodies = torch.from_numpy(g.bodyData.copy()).to(dev)
    cons = torch.from_numpy(g.consData.view(np.int32).copy()).to(dev)
    forces = torch.from_numpy(g.forceData.copy()).to(dev)
    d_rects = torch.from_numpy(rects.reshape(-1).copy()).to(dev)
    d_coll = torch.from_numpy(coll.view(np.int32).reshape(-1).copy()).to(dev)
    d_rng = torch.from_numpy(rng.view(np.int32).copy()).to(dev)
    params = _native.SolverParams(w.h, w.substeps, w.iterations, w.linDrag, w.angDrag,
                                  w.maxSpeed, w.maxAngSpeed)
    stream = torch.cuda.current_stream().cuda_stream
    for call in range(2):
        gpuworld.step(g)
        ref_b = np.zeros(nB * 12, dtype=np.float32)
        ref_c = np.zeros(nC * 20, dtype=np.uint32)
        _native.check(L.kr_download(g.handle, ref_b.ctypes.data_as(_F32P),
                                    ref_c.ctypes.data_as(_U32P)), g.handle)
        rc = L.kr_step_noalloc(C.byref(params), nB, nC, bodies.data_ptr(), cons.data_ptr(),
                               forces.data_ptr(), d_rects.data_ptr(), nR, d_coll.data_ptr(), nP,
                               d_rng.data_ptr(), 1, stream)
        assert rc == _native.KR_OK, f"call {call}: status {rc}"
        torch.cuda.synchronize()
        got_b = bodies.cpu().numpy()
        got_c = cons.cpu().numpy().view(np.uint32)
        assert np.array_equal(got_b.view(np.uint32), ref_b.view(np.uint32)), f"call {call}: bodies"
        assert np.array_equal(got_c, ref_c), f"call {call}: constraints"
    gpuworld.destroy(g)


def test_no_alloc_rejects_worlds_above_its_limits():
    L = _bind()
    params = _native.SolverParams(1 / 120, 2, 4, 3.0, 3.0, 360.0, 18.0)
    fake = C.c_void_p(16)  # never dereferenced: the size check comes first
    rc = L.kr_step_noalloc(C.byref(params), 4096, 10, fake, fake, fake, fake, 4, fake, 10,
                           fake, 1, None)
    assert rc == _native.KR_ERR_CAPACITY
    rc = L.kr_step_noalloc(C.byref(params), 10, 100000, fake, fake, fake, fake, 4, fake, 10,
                           fake, 1, None)
    assert rc == _native.KR_ERR_CAPACITY


def _dev(a, dtype=None):
    import torch
    a = np.ascontiguousarray(a)
    if dtype is not None:
        a = a.view(dtype)
    return torch.from_numpy(a.copy()).to(torch.device("cuda", 0))


def test_no_alloc_sixty_four_creatures_ten_steps_per_call_vs_f32_oracle():
    """64 creatures (4 arms x 5 segments: 1,344 bodies, 2,816 constraints,
    3,072 collision points, within the limits) advanced 10 env steps per
    call, two calls in a row, against the f32 oracle stepped the same way
    (controls held over each call, as n_steps > 1 holds them).  Bar: <= 4 ulp
    per coordinate after the first step's worth; the kernel follows the
    oracle's op order, so the test also records that it is bit-identical."""
    import torch

    L = _bind()
    seed, n, arms, segs = 11, 64, 4, 5
    ctl = [ControlStream(arms, segs, seed=200 + c).at(0) for c in range(n)]
    w, g, rects, coll, rng = _world(seed, n, arms, segs, controls=ctl)
    o = ob.Sim(seed=seed, creatures=n, arms=arms, segs=segs)
    o.world.f32ify()
    o.world.round_state()
    for c in range(n):
        o.apply_control_motors(c, TONE, *ctl[c])
    nB, nC, nP, nR = w.n, len(w.constraints), len(w.collPts), len(rects)
    assert nB <= 2048 and nC <= 4096 and nP <= 4096
    bodies = _dev(g.bodyData)
    cons = _dev(g.consData, np.int32)
    forces = _dev(g.forceData)
    d_rects = _dev(rects.reshape(-1))
    d_coll = _dev(coll.reshape(-1), np.int32)
    d_rng = _dev(rng, np.int32)
    gpuworld.destroy(g)
    params = _native.SolverParams(w.h, w.substeps, w.iterations, w.linDrag, w.angDrag,
                                  w.maxSpeed, w.maxAngSpeed)
    stream = torch.cuda.current_stream().cuda_stream
    for call in range(2):
        rc = L.kr_step_noalloc(C.byref(params), nB, nC, bodies.data_ptr(), cons.data_ptr(),
                               forces.data_ptr(), d_rects.data_ptr(), nR, d_coll.data_ptr(), nP,
                               d_rng.data_ptr(), 10, stream)
        assert rc == _native.KR_OK, f"call {call}: status {rc}"
        for _ in range(10):
            o.step32()
        torch.cuda.synchronize()
        bd = bodies.cpu().numpy().reshape(nB, 12)
        worst = 0
        for name, col in (("px", 0), ("py", 1), ("vx", 4), ("vy", 5), ("ang", 6), ("av", 8)):
            u = ulp_distance(bd[:, col], o.world.arr(name).astype(np.float32))
            worst = max(worst, int(u.max()))
            assert u.max() <= 4, f"call {call}: {name} {int(u.max())} ulp"
        assert worst == 0, f"call {call}: not bit-identical (max {worst} ulp)"
        # the grip multipliers and flags the oracle holds after its break test
        cu = cons.cpu().numpy().view(np.uint32).reshape(nC, 20)
        assert np.array_equal(cu[:, 17] != 0, np.array([bool(c.broken) for c in o.world.constraints])), \
            f"call {call}: broken flags"


def _reject(L, nB, nC, bodies, cons, coll_range, n_coll_pts=0):
    """Calls the step with small host-built worlds that the schedule builder
    must refuse; returns the status and whether the caller's bodies and
    constraints came back unchanged."""
    import torch

    params = _native.SolverParams(1 / 120, 2, 4, 3.0, 3.0, 360.0, 18.0)
    rects = np.array([0.0, 0.0, 10.0, 10.0], np.float32)
    coll = np.zeros((max(n_coll_pts, 1), 4), np.float32)
    coll[:, 3] = 1.0
    d_b, d_c, d_f = _dev(bodies), _dev(cons, np.int32), _dev(np.zeros(4 * nB, np.float32))
    d_r, d_p, d_rng = _dev(rects), _dev(coll.reshape(-1), np.int32), _dev(coll_range, np.int32)
    rc = L.kr_step_noalloc(C.byref(params), nB, nC, d_b.data_ptr(), d_c.data_ptr(), d_f.data_ptr(),
                           d_r.data_ptr(), 1, d_p.data_ptr() if n_coll_pts else None, n_coll_pts,
                           d_rng.data_ptr(), 1, torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    same = (np.array_equal(d_b.cpu().numpy().view(np.uint32), bodies.view(np.uint32)) and
            np.array_equal(d_c.cpu().numpy().view(np.uint32), cons.view(np.uint32)))
    return rc, same


def _chain(nB):
    """nB bodies in a line, joined by nB - 1 pins (one connected island)."""
    bodies = np.zeros((nB, 12), np.float32)
    bodies[:, 0] = 100 + 10 * np.arange(nB)
    bodies[:, 1] = 100
    bodies[:, 2:4] = bodies[:, 0:2]
    bodies[:, 9] = 1.0
    bodies[:, 10] = 1.0
    cons = np.zeros((max(nB - 1, 1), 20), np.float32)
    cu = cons.view(np.uint32)
    for k in range(nB - 1):
        cu[k, 0], cu[k, 1], cu[k, 2] = k, k + 1, 0
        cons[k, 4], cons[k, 6] = 5.0, -5.0
        cons[k, 16] = 1e30
    return bodies.reshape(-1), cons.reshape(-1)


def test_no_alloc_device_side_rejections_leave_buffers_untouched():
    L = _bind()
    # a constraint whose second body is past the world: KR_ERR_INDEX
    bodies, cons = _chain(2)
    cons.view(np.uint32)[1] = 5
    rc, same = _reject(L, 2, 1, bodies, cons, np.zeros(4, np.uint32))
    assert rc == _native.KR_ERR_INDEX and same
    # collRange offsets with a gap: KR_ERR_INVALID
    bodies, cons = _chain(2)
    rc, same = _reject(L, 2, 1, bodies, cons, np.array([0, 2, 1, 1], np.uint32), n_coll_pts=2)
    assert rc == _native.KR_ERR_INVALID and same
    # counts whose 32-bit sum wraps to the point count (0xffffffff + 2 = 1):
    # refused before any range is used
    rc, same = _reject(L, 2, 1, bodies, cons, np.array([0, 0xFFFFFFFF, 0xFFFFFFFF, 2], np.uint32),
                       n_coll_pts=1)
    assert rc == _native.KR_ERR_INVALID and same
    # one creature of 161 bodies, above KR_MAX_ISLAND_BODIES (160): KR_ERR_CAPACITY
    bodies, cons = _chain(161)
    rc, same = _reject(L, 161, 160, bodies, cons, np.zeros(2 * 161, np.uint32))
    assert rc == _native.KR_ERR_CAPACITY and same
    # and a valid world right after the refusals still steps (the shared
    # scratch holds nothing a later call depends on)
    bodies, cons = _chain(3)
    rc, same = _reject(L, 3, 2, bodies, cons, np.zeros(6, np.uint32))
    assert rc == _native.KR_OK
