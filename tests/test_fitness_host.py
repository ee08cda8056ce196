"""The oracle's fitness restatement (postStep accumulators, measureReach and
score of src/sim/core.js:297-356 and src/sim/fitness.js:74-172) on the CPU:
score against an independent Python restatement of scoreTerms/score, and
measureReach properties."""
import math

import numpy as np

from oracle import binding as ob


def _score_py(c):
    """scoreTerms + score (fitness.js:115-172) without prey, opts {}."""
    steps = max(1, c["steps"])
    path, disp = c["pathLen"], c["maxDisplacement"]
    reach = c["spawnReach"] if c["spawnReach"] > 0 else 300
    reach_frac = min(1.2, disp / reach)
    directed = min(1, disp / path) if path > 1 else 0
    spin_budget = steps * 18 * (1 / 60)
    heading_hold = 1 - min(1, c["angularAccum"] / max(1e-6, spin_budget))
    mean_speed = path / steps / 60
    efficiency = c["forwardProg"] / max(0.5, c["energySpent"] or 0.5)
    progress_base = c["gripPullProg"] * 2.6 + reach_frac * 320
    stride_frac = min(c["strides"], 60) / 60
    prog_gate = min(1, disp / max(1e-6, 0.25 * reach))
    terms = [c["gripPullProg"] * 2.6, progress_base * 0.5 * stride_frac, reach_frac * 320,
             directed * 70 * prog_gate, heading_hold * 28 * prog_gate,
             min(1, mean_speed) * 14 * prog_gate, min(20, efficiency) * 3 * prog_gate,
             -(c["angularAccum"] * 0.55 * 0.02), -(c["freeMove"] * 0.05),
             -(c["energySpent"] * 0.30), 0, 0]
    s = 0.0
    for t in terms:
        s += t
    return s if math.isfinite(s) else 0.0


def test_oracle_score_matches_restatement_of_fitness_js():
    rng = np.random.default_rng(0)
    for _ in range(200):
        m = ob.Metrics()
        m.steps = float(rng.integers(0, 2000))
        m.pathLen = float(rng.uniform(0, 800))
        m.maxDisplacement = float(rng.uniform(0, 300))
        m.spawnReach = float(rng.choice([0.0, rng.uniform(70, 400)]))
        m.angularAccum = float(rng.uniform(0, 60))
        m.forwardProg = float(rng.uniform(0, 400))
        m.gripPullProg = float(rng.uniform(0, 200))
        m.freeMove = float(rng.uniform(0, 100))
        m.energySpent = float(rng.choice([0.0, rng.uniform(0, 40)]))
        m.strides = float(rng.integers(0, 120))
        want = _score_py({f: getattr(m, f) for f in ob.METRIC_FIELDS})
        assert ob.lib().or_score(m) == want


def test_measure_reach_open_space_and_walls():
    box = np.array([[0, 0, 1000, 10], [0, 990, 1000, 10], [0, 0, 10, 1000], [990, 0, 10, 1000]], float)
    open_ = ob.measure_reach(box, 118.5, 500, 500)
    near = ob.measure_reach(box, 118.5, 30, 500)
    # 3.5 reaches = 414.75 px: every ray runs out in the open, 35 full steps
    assert open_ == 35 * 12
    assert 70 <= near < open_
    # a longer body reaches farther: rays run up to 3.5 of its reaches
    assert ob.measure_reach(box, 24 + 9 * 13.5, 500, 500) > open_


def test_post_step_counts_steps_and_path():
    sim = ob.Sim(seed=1, creatures=1)
    for _ in range(5):
        sim.pre_step()
        sim.step()
        sim.post_step()
    m = sim.metrics(0)
    assert m["steps"] == 5 and m["pathLen"] >= 0 and m["energySpent"] > 0
