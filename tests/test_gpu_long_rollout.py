"""Long rollouts against the FP64 oracle by fitness distributions.

The dynamics are chaotic: after a few hundred steps the f32 GPU trajectory
and the f64 oracle trajectory of the same creature part ways (the
reference measured this with its chaos checks), so long rollouts are
compared as populations, on the quantity ES selects by: the reference's
fitness score (src/sim/fitness.js:115-172, the engine's on-device
postStep accumulators and score) -- and on the mantle's path length and
net displacement.  Every creature is driven the same way on both sides
(its control stream, applyControl with the suction-cup reflex, step,
postStep); the oracle runs each creature in its own FP64 world on the
host's threads (oracle/xpbd_bench.c).  Bars: mean score within 2 %,
two-sample KS p > 0.05 for score, path length and displacement.

  * config-1 creatures: 256 default bodies on map seed 1 (spawn jitter
    +-20 px, heading U[0, 2 pi)), 600 env steps;
  * the mixed workload: 512 creatures of 4-8 arms x 5-9 segments on 16 maps,
    horizons U{300..900}."""
import os

import numpy as np
import pytest
from scipy import stats

from kraken_3_gpu_b200 import batch, workloads
from oracle import binding as ob

pytestmark = pytest.mark.gpu
F = batch.METRIC_FIELDS


def _gpu(w):
    eng = batch.BatchEngine(w.maps, w.n)
    workloads.spawn_all(eng, w)
    eng.run(int(w.horizon.max()))
    m = eng.read_metrics()
    eng.close()
    return m[:, F.index("score")], m[:, F.index("pathLen")], m[:, F.index("x")], m[:, F.index("y")]


def _oracle(w):
    _, _, out = ob.bench_rollouts(w.maps, w.map_id, w.arms, w.segs, w.x, w.y, w.angle, w.seed, w.horizon,
                                  max(1, os.cpu_count() or 1), metrics=True)
    return out[:, 3], out[:, 2], out[:, 0], out[:, 1]


def _compare(w, label):
    g_score, g_path, gx, gy = _gpu(w)
    o_score, o_path, ox, oy = _oracle(w)
    g_disp, o_disp = np.hypot(gx - w.x, gy - w.y), np.hypot(ox - w.x, oy - w.y)
    assert np.all(np.isfinite(g_score)) and np.all(g_path > 0)
    rel = abs(g_score.mean() - o_score.mean()) / abs(o_score.mean())
    p = {k: stats.ks_2samp(a, b, method="asymp").pvalue
         for k, a, b in (("score", g_score, o_score), ("path", g_path, o_path), ("disp", g_disp, o_disp))}
    print(f"{label}: mean score GPU {g_score.mean():.3f} oracle {o_score.mean():.3f} ({100 * rel:.3f} %), "
          f"mean path {g_path.mean():.2f} / {o_path.mean():.2f} px, KS p " +
          ", ".join(f"{k} {v:.3f}" for k, v in p.items()))
    assert rel < 0.02, f"mean score differs by {100 * rel:.2f} %"
    for k, v in p.items():
        assert v > 0.05, f"KS p of {k} = {v:.4f}"


def test_600_step_es_fitness_distribution_vs_fp64_oracle():
    _compare(workloads.uniform(n=256, steps=600), "config-1 creatures x 600 steps")


def test_mixed_bodies_es_fitness_distribution_vs_fp64_oracle():
    _compare(workloads.uneven(n=512, n_maps=16, seed=7, h_min=300, h_max=900), "mixed workload, 512 creatures")
