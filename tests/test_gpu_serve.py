"""GPU tests of the rollout server: device eps, weights, results alone vs in
the mix, queued admission under an HBM budget, repeatability -- under both
schedulers: two partitions in alternating rounds (slice_ms = 0) and one
partition in preemptible slices (slice_ms > 0; small slices here, so that
slices are cut by arrivals and by time; completions found by polling while
a slice runs)."""
import numpy as np
import pytest

from kraken_3_gpu_b200 import batch, serve, workloads
from tests import serve_ref

pytestmark = pytest.mark.gpu


def _maps():
    return workloads.uneven(n=4, n_maps=6, seed=11, h_min=10, h_max=20).maps


def _spawn_xy(maps, m):
    """A free spot of map m (the workload builder's spawn rule)."""
    w = workloads.uneven(n=64, n_maps=len(maps), seed=11, h_min=10, h_max=20)
    i = int(np.flatnonzero(w.map_id == m)[0])
    return float(w.x[i]), float(w.y[i])


def _requests(maps, seed=0, n=12, pop_max=24, h_max=150):
    rng = np.random.default_rng(seed)
    reqs = []
    for k in range(n):
        arms, segs = int(rng.integers(4, 9)), int(rng.integers(5, 10))
        m = int(rng.integers(0, len(maps)))
        x, y = _spawn_xy(maps, m)
        policy = k % 3 != 2
        theta = rng.normal(0, 0.1, serve.policy_params(arms, segs)).astype(np.float32) if policy else None
        reqs.append(dict(population=2 * int(rng.integers(1, pop_max // 2 + 1)),
                         horizon=int(rng.integers(40, h_max)), arms=arms, segs=segs, map_id=m,
                         x=x, y=y, angle=float(rng.uniform(0, 2 * np.pi)), theta=theta,
                         sigma=0.02, seed=int(rng.integers(0, 2**63))))
    return reqs


def test_device_eps_matches_restatement():
    for seed, pair in ((0, 0), (12345, 7), (2**63 + 5, 300)):
        got = serve.policy_eps(seed, pair, 2000)
        want = serve_ref.eps(seed, pair, 2000)
        assert np.allclose(got, want, rtol=2e-7, atol=1e-7)


def test_server_equals_engine_with_explicit_mirrored_weights():
    maps = _maps()
    arms, segs, pop, H = 6, 7, 6, 90
    x, y = _spawn_xy(maps, 2)
    rng = np.random.default_rng(5)
    n_par = serve.policy_params(arms, segs)
    theta = rng.normal(0, 0.1, n_par).astype(np.float32)
    sigma, seed = 0.05, 99
    srv = serve.Server(maps, 1 << 30, max_slots=64, chunk_steps=16)
    rid = srv.submit(pop, H, arms, segs, 2, x, y, 0.7, theta=theta, sigma=sigma, seed=seed)
    srv.drain()
    got = srv.result(rid, pop)["results"]
    srv.close()
    W = np.stack([serve_ref.mirrored_weights(theta, sigma, serve.policy_eps(seed, i // 2, n_par),
                                             1 if i % 2 == 0 else -1) for i in range(pop)])
    eng = batch.BatchEngine(maps, pop, control="policy")
    eng.spawn(0, [arms] * pop, [segs] * pop, [2] * pop, [x] * pop, [y] * pop, [0.7] * pop, [H] * pop)
    eng.set_policy(W, np.arange(pop, dtype=np.int32))
    eng.run(H)
    want = eng.read_metrics()
    eng.close()
    assert np.array_equal(got, want)
    assert not np.array_equal(got[0], got[1])  # the mirrored pair differs


MODES = [dict(slice_ms=0.0, chunk=16), dict(slice_ms=1.0, chunk=1 << 20)]


def _run(maps, reqs, max_slots, stagger=0.0, chunk=16, obs_ring=0, slice_ms=0.0):
    srv = serve.Server(maps, 2 << 30, max_slots=max_slots, chunk_steps=chunk, obs_ring=obs_ring,
                       slice_ms=slice_ms)
    t0 = srv.now() + 0.01
    ids = [srv.submit(**r, arrival=t0 + k * stagger) for k, r in enumerate(reqs)]
    srv.drain()
    out = [srv.result(i, r["population"]) for i, r in zip(ids, reqs)]
    st = srv.stats()
    srv.close()
    return out, st


@pytest.mark.parametrize("mode", MODES)
def test_each_request_same_alone_and_in_the_mix(mode):
    maps = _maps()
    reqs = _requests(maps)
    alone = [_run(maps, [r], max_slots=64, **mode)[0][0] for r in reqs]
    mixed, st = _run(maps, reqs, max_slots=96, stagger=0.004, **mode)
    assert st["completed"] == len(reqs)
    for a, m in zip(alone, mixed):
        assert np.array_equal(a["results"], m["results"])
    # continuous batching: a request admitted while an earlier one was running
    overlap = any(mixed[j]["admitted"] > mixed[i]["admitted"] and mixed[j]["admitted"] < mixed[i]["completed"]
                  for i in range(len(reqs)) for j in range(len(reqs)))
    assert overlap
    for m in mixed:
        assert m["arrival"] <= m["admitted"] <= m["completed"]


@pytest.mark.parametrize("mode", MODES)
def test_queued_admission_under_budget_bit_identical_three_runs(mode):
    maps = _maps()
    reqs = _requests(maps, seed=3, n=16, pop_max=16, h_max=120)
    for r in reqs:
        r["theta"] = None  # control streams, as the memory-bound configuration
    budget_slots = 32
    runs = [_run(maps, reqs, max_slots=budget_slots, obs_ring=128, **mode) for _ in range(3)]
    total = sum(r["population"] for r in reqs)
    assert total > budget_slots
    for out, st in runs:
        assert st["capacity"] == budget_slots and st["completed"] == len(reqs)
        # some request waited for slots
        assert max(o["admitted"] - o["arrival"] for o in out) > 0
    for out, _ in runs[1:]:
        for a, b in zip(runs[0][0], out):
            assert np.array_equal(a["results"], b["results"])


def test_server_rejects_bad_requests():
    maps = _maps()
    srv = serve.Server(maps, 1 << 30, max_slots=16)
    from kraken_3_gpu_b200 import _native
    with pytest.raises(_native.KrError):
        srv.submit(10, 50, 6, 7, 0, 100, 100, 0)  # more than a partition (8)
    with pytest.raises(_native.KrError):
        srv.submit(2, 50, 6, 7, 99, 100, 100, 0)  # unknown map
    with pytest.raises(_native.KrError):
        srv.submit(2, 50, 6, 7, 0, 100, 100, 0, theta=np.zeros(10, np.float32))
    srv.close()


@pytest.mark.parametrize("mode", [dict(slice_ms=0.0, chunk_steps=24), dict(slice_ms=0.5, chunk_steps=1 << 20),
                                  dict(slice_ms=1000.0, chunk_steps=1 << 20)])
def test_served_uneven_workload_equals_batched_engine(mode):
    """The mixed workload submitted as requests (one per creature, its own
    pose, control stream and horizon) gives the batched engine's results --
    with slices cut every half millisecond, and with slices that run until
    an arrival fits (a creature's slot frees only when its slice ends)."""
    w = workloads.uneven(n=60, n_maps=5, seed=13, h_min=30, h_max=120)
    eng = batch.BatchEngine(w.maps, w.n)
    workloads.spawn_all(eng, w)
    eng.run(int(w.horizon.max()))
    want = eng.read_metrics()
    eng.close()
    srv = serve.Server(w.maps, 1 << 30, max_slots=40, policy=False, **mode)
    half = w.n // 2
    ids = []
    for i in range(half):  # one call per request
        ids.append(srv.submit(1, int(w.horizon[i]), int(w.arms[i]), int(w.segs[i]), int(w.map_id[i]),
                              xs=[w.x[i]], ys=[w.y[i]], angles=[w.angle[i]], control_seeds=[w.seed[i]]))
    s = slice(half, w.n)  # the rest in one batch call
    ids += list(srv.submit_many(w.horizon[s], w.arms[s], w.segs[s], w.map_id[s], w.x[s], w.y[s],
                                w.angle[s], control_seeds=w.seed[s]))
    srv.drain()
    got = np.concatenate([srv.result(r, 1)["results"] for r in ids[:half]])
    rest, times = srv.results_many(ids[half:], release=True)
    srv.close()
    assert np.array_equal(np.concatenate([got, rest]), want)
    assert np.all(times[:, 0] <= times[:, 1]) and np.all(times[:, 1] <= times[:, 2])


def test_sliced_requests_complete_while_their_slice_runs():
    """Slices: a short request completes (its records copied back beside the
    running kernel) while the slice that runs it still runs a long one --
    one slice in all, its time (10 s) longer than the run -- and every
    request's results equal the batched engine's.  A request released while
    its slice still holds its slots is gone for the caller at once and is
    freed when the slice ends."""
    import time

    from kraken_3_gpu_b200 import _native

    w = workloads.uneven(n=6, n_maps=2, seed=17, h_min=20, h_max=30)
    w.horizon[0] = 3000  # the long request
    eng = batch.BatchEngine(w.maps, w.n)
    workloads.spawn_all(eng, w)
    eng.run(int(w.horizon.max()))
    want = eng.read_metrics()
    eng.close()
    srv = serve.Server(w.maps, 1 << 30, max_slots=8, policy=False, slice_ms=10000.0, chunk_steps=1 << 20)
    ids = list(srv.submit_many(w.horizon, w.arms, w.segs, w.map_id, w.x, w.y, w.angle, control_seeds=w.seed))
    early = None
    released = None
    t_end = time.monotonic() + 60
    while time.monotonic() < t_end:
        busy = srv.pump()
        done = set(srv.poll())
        if done and early is None:
            early = (srv.stats(), done)
            released = min(done)
            kept = srv.result(released, 1)["results"]
            srv.release(released)  # its slice still runs and holds its slot
            with pytest.raises(_native.KrError):
                srv.result(released, 1)
        if not busy:
            break
        time.sleep(0.0002)
    srv.drain()
    others = [i for i in ids if i != released]
    rest, times = srv.results_many(others, release=True)
    st = srv.stats()
    srv.close()
    assert early is not None
    first_stats, first_done = early
    assert ids[0] not in first_done and first_stats["rounds"] == 1
    assert st["rounds"] == 1 and st["completed"] == w.n  # the one slice ran every request
    k = ids.index(released)
    assert np.array_equal(kept, want[k:k + 1])
    assert np.array_equal(rest, np.delete(want, k, axis=0))
    assert times[others.index(ids[0]), 2] == times[:, 2].max()


def test_sliced_server_closes_without_running_its_slice_out():
    """Destroying a server with a slice in flight stops the slice at its
    creatures' next env step: closing takes a small fraction of the time the
    running request needs (100,000 env steps)."""
    import time

    w = workloads.uneven(n=8, n_maps=2, seed=19, h_min=20, h_max=30)
    srv = serve.Server(w.maps, 1 << 30, max_slots=8, policy=False, slice_ms=10000.0, chunk_steps=1 << 20)
    srv.submit_many(np.full(w.n, 100000, np.int32), w.arms, w.segs, w.map_id, w.x, w.y, w.angle,
                    control_seeds=w.seed)
    srv.pump()  # admits and launches the slice
    time.sleep(0.05)
    t0 = time.monotonic()
    srv.close()
    assert time.monotonic() - t0 < 1.0
