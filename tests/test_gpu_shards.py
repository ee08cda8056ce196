"""The multi-GPU partitioning on one GPU: shards of one workload run one
after the other in separate engines (as separate ranks would run them) give
the unsharded run's results bit for bit, and a mirrored ES population split
over two servers by pair ranges (first_individual) gives the whole
population's results bit for bit -- so N ranks' gathered results equal one
rank's run of the same creatures."""
import numpy as np
import pytest

from kraken_3_gpu_b200 import batch, replicas, serve, workloads

pytestmark = pytest.mark.gpu


def _run(w):
    eng = batch.BatchEngine(w.maps, w.n)
    workloads.spawn_all(eng, w)
    eng.run(int(w.horizon.max()))
    m = eng.read_metrics()
    st = eng.read_state()
    eng.close()
    return m, st


@pytest.mark.parametrize("world", [2, 3])
def test_workload_shards_equal_the_whole_run(world):
    w = workloads.uneven(n=96, n_maps=4, seed=21, h_min=40, h_max=90)
    full_m, _ = _run(w)
    parts = []
    for r in range(world):
        sw, (lo, hi) = replicas.shard(w, r, world, balance=True)
        assert sw.n == hi - lo > 0
        parts.append(_run(sw)[0])
    got = np.concatenate(parts)
    assert np.array_equal(got.view(np.uint64), full_m.view(np.uint64))


def _spawn_xy(maps, m):
    w = workloads.uneven(n=64, n_maps=len(maps), seed=11, h_min=10, h_max=20)
    i = int(np.flatnonzero(w.map_id == m)[0])
    return float(w.x[i]), float(w.y[i])


@pytest.mark.parametrize("with_theta", [True, False])
def test_population_split_over_servers_equals_the_whole(with_theta):
    maps = workloads.uneven(n=4, n_maps=4, seed=11, h_min=10, h_max=20).maps
    arms, segs, pop, H = 5, 6, 22, 70
    x, y = _spawn_xy(maps, 1)
    rng = np.random.default_rng(3)
    theta = rng.normal(0, 0.1, serve.policy_params(arms, segs)).astype(np.float32) if with_theta else None
    kw = dict(theta=theta, sigma=0.03, seed=4242)
    whole = serve.Server(maps, 1 << 30, max_slots=64, chunk_steps=16, policy=with_theta)
    rid = whole.submit(pop, H, arms, segs, 1, x, y, 0.3, **kw)
    whole.drain()
    ref = whole.result(rid, pop)["results"]
    whole.close()
    pieces = []
    world = 2
    for r in range(world):  # one server per rank, run one after the other
        first, count = replicas.pair_range(pop, r, world)
        srv = serve.Server(maps, 1 << 30, max_slots=64, chunk_steps=16, policy=with_theta)
        q = srv.submit(count, H, arms, segs, 1, x, y, 0.3, first_individual=first, **kw)
        srv.drain()
        pieces.append(srv.result(q, count)["results"])
        srv.close()
    got = np.concatenate(pieces)
    assert got.shape == ref.shape
    assert np.array_equal(got.view(np.uint64), ref.view(np.uint64))
