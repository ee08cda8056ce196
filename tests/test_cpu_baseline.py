"""The timed CPU baseline (oracle/xpbd_bench.c) computes what the engine
computes: each creature driven by its control stream, applyControl with
the reflex, the FP64 step and postStep.  Its C loop on POSIX threads must
give the same final mantle positions and path lengths as the same oracle
driven step by step from Python, bit for bit, whatever the thread count."""
import numpy as np

from kraken_3_gpu_b200 import workloads
from kraken_3_gpu_b200.kraken import arm_reach
from kraken_3_gpu_b200.workloads import TONE, ControlStream
from oracle import binding as ob


def _python_loop(w, i, steps):
    s = ob.Sim(rects=w.maps[w.map_id[i]])
    s.add_creature(w.x[i], w.y[i], w.angle[i], int(w.arms[i]), int(w.segs[i]))
    s.set_spawn_reach(0, ob.measure_reach(w.maps[w.map_id[i]], arm_reach(int(w.segs[i])), w.x[i], w.y[i]))
    cs = ControlStream(int(w.arms[i]), int(w.segs[i]), seed=int(w.seed[i]))
    for t in range(steps):
        tg, ad = (v.astype(np.float32).astype(np.float64) for v in cs.at(t))
        s.apply_control_motors(0, TONE, tg, ad)
        s.pre_step()
        s.step()
        s.post_step()
    m = s.metrics(0)
    return m["x"], m["y"], m["pathLen"], m["score"]


def test_threaded_c_loop_equals_python_driven_oracle():
    w = workloads.uneven(n=64, n_maps=4, seed=5, h_min=30, h_max=45)
    sel = np.arange(0, 64, 8)
    ref = np.array([_python_loop(w, i, int(w.horizon[i])) for i in sel])
    for threads in (1, 3):
        steps, el, out = ob.bench_rollouts(w.maps, w.map_id[sel], w.arms[sel], w.segs[sel], w.x[sel],
                                           w.y[sel], w.angle[sel], w.seed[sel], w.horizon[sel], threads,
                                           metrics=True)
        assert steps == int(w.horizon[sel].sum()) and el > 0
        assert np.array_equal(out, ref), f"{threads} threads"


def test_time_limit_stops_early():
    w = workloads.uneven(n=16, n_maps=2, seed=6, h_min=100000, h_max=100000)
    steps, el = ob.bench_rollouts(w.maps, w.map_id, w.arms, w.segs, w.x, w.y, w.angle, w.seed, w.horizon,
                                  2, limit_s=0.3)
    assert 0 < steps < 16 * 100000 and el < 5.0
