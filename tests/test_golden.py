"""The oracle against the committed golden fixtures (tests/golden, made by
tests/golden/make_golden.py): bit for bit, on the CPU."""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
import make_golden  # noqa: E402


def _load(name):
    return dict(np.load(os.path.join(HERE, "golden", name)))


def test_oracle_reproduces_config0_fixtures():
    for f32, name in ((False, "config0_f64.npz"), (True, "config0_f32.npz")):
        want = _load(name)
        got = make_golden.config0(f32)
        assert sorted(got) == sorted(want)
        for k in want:
            assert np.array_equal(got[k], want[k]), (name, k)
    # the scenario exercises the suction cups: attach and release events
    g = _load("config0_f64.npz")["grips"]
    assert (g[:, 0] != g[:, 1]).any() or (g[1:, 0] != g[:-1, 1]).any()


def test_oracle_reproduces_batch_fixture():
    want = _load("batch_f32.npz")
    got = make_golden.batch()
    for k in want:
        assert np.array_equal(got[k], want[k]), k


def test_fixtures_are_finite_and_moving():
    g = _load("config0_f32.npz")
    assert np.all(np.isfinite(g["px_60"])) and not np.array_equal(g["px_1"], g["px_60"])
