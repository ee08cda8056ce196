"""The engine's on-device fitness metrics (postStep and score) against the
f32 oracle driven like the reference's trainer loop (applyControl, preStep,
step, postStep), creature by creature; and the server's results."""
import numpy as np
import pytest

from kraken_3_gpu_b200 import batch, kraken, serve, workloads
from oracle import binding as ob
from tests.scenarios import TONE, ControlStream

pytestmark = pytest.mark.gpu
INT_FIELDS = ("steps", "anchoredSteps", "gripCycles", "strides", "attachEvents")


def _oracle_metrics(w, i, steps):
    rects32 = w.maps[w.map_id[i]].astype(np.float32).astype(np.float64)
    sim = ob.Sim(rects=rects32)
    sim.add_creature(w.x[i], w.y[i], w.angle[i], int(w.arms[i]), int(w.segs[i]))
    sim.world.f32ify()
    sim.world.round_state()
    sim.set_spawn_reach(0, ob.measure_reach(rects32, kraken.arm_reach(int(w.segs[i])), w.x[i], w.y[i]))
    cs = ControlStream(int(w.arms[i]), int(w.segs[i]), seed=int(w.seed[i]))
    for s in range(steps):
        t, a = cs.at(s)
        sim.apply_control_motors(0, TONE, t, a)
        sim.pre_step()
        sim.step32()
        sim.post_step()
    return sim.metrics(0)


def test_engine_metrics_equal_oracle_post_step_and_score():
    w = workloads.uneven(n=24, n_maps=4, seed=5, h_min=60, h_max=60)
    eng = batch.BatchEngine(w.maps, w.n)
    workloads.spawn_all(eng, w)
    eng.run(60)
    got = eng.read_metrics()
    eng.close()
    anchored_any = 0
    for i in range(w.n):
        want = _oracle_metrics(w, i, 60)
        for j, f in enumerate(batch.METRIC_FIELDS):
            if f in INT_FIELDS:
                assert got[i, j] == want[f], (i, f)
            else:
                assert np.isclose(got[i, j], want[f], rtol=1e-10, atol=1e-9), (i, f, got[i, j], want[f])
        anchored_any += want["anchoredSteps"] > 0
    assert anchored_any > 0  # the scenario exercises the suction cups


def test_server_results_are_the_metrics_record():
    w = workloads.uneven(n=16, n_maps=3, seed=6, h_min=40, h_max=90)
    eng = batch.BatchEngine(w.maps, w.n)
    workloads.spawn_all(eng, w)
    eng.run(int(w.horizon.max()))
    want = eng.read_metrics()
    eng.close()
    srv = serve.Server(w.maps, 1 << 30, max_slots=16, chunk_steps=32, policy=False)
    ids = srv.submit_many(w.horizon, w.arms, w.segs, w.map_id, w.x, w.y, w.angle, control_seeds=w.seed)
    srv.drain()
    got, _ = srv.results_many(ids, release=True)
    srv.close()
    assert got.shape == (w.n, serve.RESULT_WORDS)
    assert np.array_equal(got, want)
    assert np.all(got[:, 1] == w.horizon)  # steps


def test_spawn_reach_bit_exact_on_many_maps():
    """measureReach runs in the spawn kernel; it equals the oracle's f64 march
    exactly, creature by creature, over 64 maps of varying density."""
    w = workloads.uneven(n=2048, n_maps=64, seed=9, h_min=1, h_max=1)
    eng = batch.BatchEngine(w.maps, w.n)
    workloads.spawn_all(eng, w)
    got = eng.read_metrics()[:, batch.METRIC_FIELDS.index("spawnReach")]
    eng.close()
    for i in range(w.n):
        rects32 = w.maps[w.map_id[i]].astype(np.float32).astype(np.float64)
        want = ob.measure_reach(rects32, kraken.arm_reach(int(w.segs[i])), w.x[i], w.y[i])
        assert got[i] == want, (i, got[i], want)
