"""GPU paths against the committed golden fixtures (tests/golden): the
drop-in driven like the reference's hybrid loop, and the batched engine."""
import os

import numpy as np
import pytest

from kraken_3_gpu_b200 import batch, workloads
from tests.scenarios import TONE, ControlStream, ulp_distance
from tests.test_gpu_parity import Hybrid

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
FIELDS = ("px", "py", "vx", "vy", "ang", "av")


def _load(name):
    return dict(np.load(os.path.join(HERE, "golden", name)))


def test_dropin_config0_vs_golden_fixtures():
    f32, f64 = _load("config0_f32.npz"), _load("config0_f64.npz")
    g = Hybrid(1, 1)
    try:
        cs = ControlStream(seed=0)
        grips = []
        for s in range(60):
            t, a = cs.at(s)
            g.control(0, t, a)
            before = g.grips(0)
            g.step()
            grips.append([before, g.grips(0)])
            if s + 1 in (1, 10, 60):
                n = g.w.n
                for f in FIELDS:
                    got = getattr(g.w, f)[:n].astype(np.float32)
                    u = ulp_distance(got, f32[f"{f}_{s + 1}"])
                    assert u.max() <= 4 and u.max() == 0, (f, s + 1, int(u.max()))
                d = max(np.max(np.abs(g.w.px[:n] - f64[f"px_{s + 1}"])),
                        np.max(np.abs(g.w.py[:n] - f64[f"py_{s + 1}"])))
                assert d <= (1e-3 if s == 0 else 1e-2), (s + 1, d)
        grips = np.array(grips, dtype=np.uint8)
        assert np.array_equal(grips, f32["grips"])
        assert np.array_equal(grips, f64["grips"])  # same attach / break events as FP64
    finally:
        g.close()


@pytest.mark.parametrize("lanes", [32, 16, 8])
def test_batched_engine_vs_golden_fixture(lanes):
    want = _load("batch_f32.npz")
    w = workloads.uneven(n=8, n_maps=2, seed=5, h_min=30, h_max=30)
    eng = batch.BatchEngine(w.maps, w.n)
    eng.set_launch(2, 0, lanes_per_creature=lanes)
    workloads.spawn_all(eng, w)
    eng.run(30)
    st = eng.read_state()
    eng.close()
    for f in FIELDS:
        assert np.array_equal(st[f], want[f]), f
    for i in range(w.n):
        A = int(w.arms[i])
        assert np.array_equal(st["grips"][i, :A, 3].astype(np.uint8), want["grips"][i, :A]), i
