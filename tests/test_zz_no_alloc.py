"""The allocation-free step entry point (kr_step_noalloc) against the
regular one (kr_create / kr_upload / kr_step).

Some callers cannot allocate GPU memory -- an application that owns every
device allocation through its own pool, or a latency-critical loop where a
cudaMalloc and its implicit synchronization are not allowed.  They call
kr_step_noalloc with their own device buffers; the library keeps its
scratch (the per-creature schedule) in one fixed-size device array.  This
test gives it the same world the regular entry point runs and checks that
two calls in a row produce the same bodies and constraints, bit for bit
(the tolerance of every other parity test here), and that a world above the
stated limits is rejected.  It runs last so that a failure here never hides
another test's result.
"""
import ctypes as C

import numpy as np
import pytest

from kraken_3_gpu_b200 import _native, core, gpuworld
from kraken_3_gpu_b200.workloads import TONE, ControlStream

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


def _world():
    sim = core.create_sim(seed=3, creatures=2)
    w, m = sim["world"], sim["map"]
    g = gpuworld.create(w, m)
    gpuworld.upload(g)
    gpuworld.download(g)
    for ci, c in enumerate(sim["creatures"]):
        t, a = ControlStream(seed=40 + ci).at(0)
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
