"""Long rollouts against the FP64 oracle by fitness distributions.

The dynamics are chaotic: after a few hundred steps the f32 GPU trajectory
and the f64 oracle trajectory of the same creature part ways (the
reference measured this with its chaos checks), so long rollouts are
compared as populations.  256 default creatures on map seed 1 (spawn jitter
+-20 px, heading U[0, 2 pi)), 600 env steps with control streams: the
path length of every creature's mantle on the GPU (batched engine) and in
its own one-creature FP64 oracle world, driven the same way.  Bars: mean
path length within 2 %, two-sample KS p > 0.05 for path length and for
net displacement."""
import threading

import numpy as np
import pytest
from scipy import stats

from kraken_3_gpu_b200 import batch, workloads
from oracle import binding as ob
from tests.scenarios import TONE, ControlStream

pytestmark = pytest.mark.gpu
N, STEPS = 256, 600


def _oracle_fitness(w):
    path = np.zeros(w.n)
    disp = np.zeros(w.n)

    def run(idx):
        for i in idx:
            sim = ob.Sim(rects=w.maps[0])
            k = sim.add_creature(w.x[i], w.y[i], w.angle[i])
            cs = ControlStream(6, 7, seed=int(w.seed[i]))
            m = k.mantle
            x0, y0 = sim.world.px[m], sim.world.py[m]
            lx, ly, pl = x0, y0, 0.0
            for s in range(STEPS):
                t, a = cs.at(s)
                sim.apply_control_motors(0, TONE, t, a)
                sim.step()
                x, y = sim.world.px[m], sim.world.py[m]
                pl += float(np.hypot(x - lx, y - ly))
                lx, ly = x, y
            path[i] = pl
            disp[i] = float(np.hypot(lx - x0, ly - y0))

    th = [threading.Thread(target=run, args=(range(t, w.n, 16),)) for t in range(16)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    return path, disp


def test_600_step_fitness_distribution_vs_fp64_oracle():
    w = workloads.uniform(n=N, steps=STEPS)
    eng = batch.BatchEngine(w.maps, w.n)
    workloads.spawn_all(eng, w)
    eng.run(STEPS)
    fit = eng.read_fitness()
    eng.close()
    g_path = fit[:, 0]
    g_disp = np.hypot(fit[:, 1] - w.x.astype(np.float32), fit[:, 2] - w.y.astype(np.float32))
    o_path, o_disp = _oracle_fitness(w)
    assert np.all(np.isfinite(g_path)) and np.all(g_path > 0)
    rel = abs(g_path.mean() - o_path.mean()) / o_path.mean()
    p_path = stats.ks_2samp(g_path, o_path, method="asymp").pvalue
    p_disp = stats.ks_2samp(g_disp, o_disp, method="asymp").pvalue
    print(f"mean path GPU {g_path.mean():.3f} oracle {o_path.mean():.3f} px ({100 * rel:.3f} %), "
          f"KS p path {p_path:.3f} displacement {p_disp:.3f}")
    assert rel < 0.02, f"mean path length differs by {100 * rel:.2f} %"
    assert p_path > 0.05
    assert p_disp > 0.05
