"""The reference's hybrid loop over the drop-in (host reflex on the mirrored
f32 state, uploadControls, one kr_step, download; kraken_3_gpu_b200.hybrid)
against the batched engine, which runs the same controls and reflex on the
device in one persistent launch: the same creatures (config 1's spawn rule,
their own control streams) end in the same state, bit for bit -- every body's
position, angle and velocities and every grip's flag."""
import numpy as np
import pytest

from kraken_3_gpu_b200 import batch, hybrid, workloads

pytestmark = pytest.mark.gpu


def test_hybrid_loop_through_the_dropin_equals_the_engine():
    import torch

    n, steps = 96, 150
    w = workloads.uniform(n=n, steps=steps)
    stream = torch.cuda.current_stream()
    loop = hybrid.HybridLoop(w, stream.cuda_stream)
    for _ in range(steps):
        loop.step()
    torch.cuda.synchronize()
    crs = loop.sim["creatures"]
    nb = 1 + sum(len(a.segs) for a in crs[0].arms)
    body = loop.body.reshape(n, nb, 12)  # creatures are contiguous in the world, mantle first
    flags = loop.consu[loop.grips, 17].copy()
    assert all(c.mantle == i * nb for i, c in enumerate(crs))
    loop.close()
    eng = batch.BatchEngine(w.maps, n)
    eng.set_stream(stream.cuda_stream)
    workloads.spawn_all(eng, w)
    eng.run(steps)
    st = eng.read_state()
    eng.close()
    assert np.all(st["steps"] == steps)
    for f, col in (("px", 0), ("py", 1), ("vx", 4), ("vy", 5), ("ang", 6), ("av", 8)):
        assert np.array_equal(st[f][:, :nb], body[:, :, col]), f
    assert np.array_equal(st["grips"][:, :6, 3] != 0, flags != 0)
    assert flags.any() and not flags.all()  # the suction cups attach and release
