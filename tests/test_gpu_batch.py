"""GPU parity of the batched engine (uneven bodies, several maps, device
reflex and proprioception) against the f32 oracle, creature by creature.

Each creature of the batch must equal a one-creature f32-oracle world on its
map at its spawn pose, driven by the reference's hybrid loop with the same
control stream: bit-identical body state and grip flags (the engine runs the
same f32 op sequence; reflex and proprioception are f64 on both sides), and
proprioception within 1e-6 of the oracle's readProprio.
"""
import numpy as np
import pytest

from kraken_3_gpu_b200 import batch, workloads
from oracle import binding as ob
from tests.scenarios import TONE, ControlStream

pytestmark = pytest.mark.gpu


def _small_uneven(n=24, n_maps=4, h=40):
    w = workloads.uneven(n=n, n_maps=n_maps, seed=5, h_min=h, h_max=h)
    return w


def _oracle_run(w, i, steps, record_obs=False):
    sim = ob.Sim(rects=w.maps[w.map_id[i]])
    k = sim.add_creature(w.x[i], w.y[i], w.angle[i], int(w.arms[i]), int(w.segs[i]))
    sim.world.f32ify()
    sim.world.round_state()
    cs = ControlStream(int(w.arms[i]), int(w.segs[i]), seed=int(w.seed[i]))
    obs = []
    for s in range(steps):
        if record_obs:
            obs.append(sim.read_proprio(0))
        t, a = cs.at(s)
        sim.apply_control_motors(0, TONE, t, a)
        sim.step32()
    grips = [k.grip(a).broken for a in range(int(w.arms[i]))]
    return sim, grips, obs


def test_uneven_batch_bit_exact_vs_f32_oracle():
    w = _small_uneven()
    eng = batch.BatchEngine(w.maps, w.n, obs_ring=64)
    workloads.spawn_all(eng, w)
    eng.run(40)
    st = eng.read_state()
    obs = eng.read_obs()
    assert np.all(st["steps"] == 40)
    for i in range(w.n):
        sim, grips, o_obs = _oracle_run(w, i, 40, record_obs=True)
        nb = sim.world.n
        for f in ("px", "py", "ang", "vx", "vy", "av"):
            got = st[f][i, :nb]
            ref = sim.world.arr(f).astype(np.float32)
            assert np.array_equal(got, ref), f"creature {i} ({w.arms[i]}x{w.segs[i]}) field {f}"
        assert [bool(g) for g in st["grips"][i, : int(w.arms[i]), 3]] == grips
        A = int(w.arms[i])
        for s in range(40):
            p = obs[i, s, : 6 * A + 6]
            assert np.allclose(p, o_obs[s], atol=1e-6, rtol=0), (i, s)
            flags = int(obs[i, s, batch.OBS_STRIDE - 1].view(np.uint32))
            assert flags == sum(1 << a for a in range(A) if o_obs[s][5 * A + a] == 1.0)
    eng.close()


def test_chunked_runs_and_graph_equal_one_run():
    w = _small_uneven(n=16, h=60)
    ref = batch.BatchEngine(w.maps, w.n)
    workloads.spawn_all(ref, w)
    ref.run(60)
    a = ref.read_state()
    chunked = batch.BatchEngine(w.maps, w.n)
    workloads.spawn_all(chunked, w)
    for _ in range(6):
        chunked.run(10)
    b = chunked.read_state()
    graphed = batch.BatchEngine(w.maps, w.n)
    workloads.spawn_all(graphed, w)
    graphed.run_graph(15, launches=4, replays=1)
    c = graphed.read_state()
    for f in ("px", "py", "ang", "vx", "vy", "av"):
        assert np.array_equal(a[f], b[f]) and np.array_equal(a[f], c[f]), f
    assert np.all(a["steps"] == 60) and np.all(c["steps"] == 60)
    for e in (ref, chunked, graphed):
        e.close()


@pytest.mark.parametrize("warps", [1, 4, 16])
def test_launch_shape_does_not_change_results(warps):
    w = _small_uneven(n=20, h=30)
    base = batch.BatchEngine(w.maps, w.n)
    workloads.spawn_all(base, w)
    base.run(30)
    other = batch.BatchEngine(w.maps, w.n)
    other.set_launch(warps, 1)
    workloads.spawn_all(other, w)
    other.run(30)
    s0, s1 = base.read_state(), other.read_state()
    for f in ("px", "py", "ang"):
        assert np.array_equal(s0[f], s1[f])
    base.close()
    other.close()


def test_horizons_stop_each_creature():
    w = workloads.uneven(n=12, n_maps=2, seed=9, h_min=5, h_max=25)
    eng = batch.BatchEngine(w.maps, w.n)
    workloads.spawn_all(eng, w)
    eng.run(100)
    st = eng.read_state()
    assert np.array_equal(st["steps"], w.horizon)
    assert eng.live() == 0
    eng.close()
