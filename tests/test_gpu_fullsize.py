"""Size-independent properties at the full sizes of the measured
configurations, where the oracle cannot follow (it runs ~5e4 creature-steps/s
on a whole host): determinism, launch-shape and time-slice invariance,
chunking, the served form (both schedulers) against the persistent form,
queued admission under a memory budget.
Every comparison is bit for bit."""
import numpy as np
import pytest

from kraken_3_gpu_b200 import batch, serve, workloads

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def mixed16k():
    return workloads.uneven(n=16384, n_maps=64, seed=2, h_min=200, h_max=2000)


def _state(eng):
    st = eng.read_state()
    return st, eng.read_metrics()


def test_mixed_16k_deterministic_and_shape_invariant(mixed16k):
    w = mixed16k
    eng = batch.BatchEngine(w.maps, w.n)
    workloads.spawn_all(eng, w)
    eng.snapshot()
    runs = []
    # (lanes, warps, CTAs per SM, time slice ms): the last two runs are cut
    # into 50 ms slices, regrouped between them (the automatic per-slice
    # shape in the last)
    for shape in ((8, 8, 0, 0), (8, 8, 0, 0), (16, 8, 0, 0), (32, 8, 0, 0), (8, 16, 1, 50), (0, 0, 0, 50)):
        eng.set_launch(shape[1], shape[2], lanes_per_creature=shape[0])
        eng.set_slice(shape[3])
        eng.restore()
        eng.run(int(w.horizon.max()))
        if shape[3] > 0:
            assert eng.last_slices() > 1
        runs.append(_state(eng))
    eng.close()
    st0, fit0 = runs[0]
    assert np.array_equal(st0["steps"], w.horizon)
    nb = 1 + 8 * 9
    assert np.all(np.isfinite(st0["px"][:, :nb])) and np.all(np.isfinite(fit0))
    for st, fit in runs[1:]:
        for f in ("px", "py", "ang", "vx", "vy", "av", "grips"):
            assert np.array_equal(st0[f], st[f]), f
        assert np.array_equal(fit0, fit)


SCHEDULERS = [dict(chunk_steps=64), dict(chunk_steps=1 << 20, slice_ms=50.0)]


@pytest.mark.parametrize("sched", SCHEDULERS, ids=["two_partitions", "slices"])
def test_mixed_16k_served_equals_persistent(mixed16k, sched):
    """The 16k workload as one request per creature equals the persistent
    engine's metrics under both schedulers (slices: requests completing while
    their slice runs, their records copied back beside the kernel)."""
    w = mixed16k
    eng = batch.BatchEngine(w.maps, w.n)
    workloads.spawn_all(eng, w)
    eng.run(int(w.horizon.max()))
    want = eng.read_metrics()
    eng.close()
    srv = serve.Server(w.maps, 8 << 30, max_slots=w.n, policy=False, **sched)
    ids = srv.submit_many(w.horizon, w.arms, w.segs, w.map_id, w.x, w.y, w.angle, control_seeds=w.seed)
    srv.drain()
    got, times = srv.results_many(ids, release=True)
    st = srv.stats()
    srv.close()
    assert st["completed"] == w.n
    assert np.array_equal(got, want)
    assert np.all(times[:, 2] >= times[:, 1])


def test_uniform_1024_chunked_equals_one_launch():
    w = workloads.uniform(n=1024, steps=1000)
    one = batch.BatchEngine(w.maps, w.n)
    workloads.spawn_all(one, w)
    one.run(1000)
    chunked = batch.BatchEngine(w.maps, w.n)
    workloads.spawn_all(chunked, w)
    for _ in range(8):
        chunked.run(125)
    a, b = _state(one), _state(chunked)
    for f in ("px", "py", "ang", "grips", "steps"):
        assert np.array_equal(a[0][f], b[0][f]), f
    assert np.array_equal(a[1], b[1])
    one.close()
    chunked.close()


@pytest.mark.parametrize("sched", [dict(chunk_steps=128), dict(chunk_steps=1 << 20, slice_ms=50.0)],
                         ids=["two_partitions", "slices"])
def test_65k_queued_under_budget_bit_identical_three_runs(sched):
    """65,536 mixed creatures (horizons up to 4,096, 128-step observation
    rings) through a server whose memory budget holds fewer slots than
    creatures, so requests queue for slots; three runs, same bits, under
    either scheduler."""
    w = workloads.uneven(n=65536, n_maps=64, seed=4, h_min=200, h_max=4096)
    budget = int(1.5 * (1 << 30))
    cap, per_slot = serve.plan(w.maps, budget, policy=False, obs_ring=128, **sched)
    assert cap < w.n
    out = []
    for _ in range(3):
        srv = serve.Server(w.maps, budget, policy=False, obs_ring=128, **sched)
        ids = srv.submit_many(w.horizon, w.arms, w.segs, w.map_id, w.x, w.y, w.angle, control_seeds=w.seed)
        srv.drain()
        res, times = srv.results_many(ids, release=True)
        st = srv.stats()
        srv.close()
        assert st["capacity"] == cap and st["completed"] == w.n
        assert np.max(times[:, 1] - times[:, 0]) > 0  # some requests waited for slots
        out.append(res)
    assert np.all(np.isfinite(out[0]))
    assert np.array_equal(out[0], out[1]) and np.array_equal(out[0], out[2])
