"""The multi-GPU plumbing (kraken_3_gpu_b200.replicas) with two gloo ranks on
the CPU: contiguous workload shards, barrier, max over ranks, the whole-job
rate, the partition / gather of an ES generation, and a rank that times out
instead of hanging."""
import os
import socket

import numpy as np
import torch.multiprocessing as mp


def _port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK="0")
    from kraken_3_gpu_b200 import replicas, workloads
    r, wsz, _ = replicas.dist_env()
    replicas.init("gloo", wsz, timeout_s=30)
    w_all = workloads.uneven(n=64, n_maps=2, seed=2, h_min=10, h_max=20)
    w, _ = replicas.shard(w_all, r, wsz)
    replicas.barrier(wsz, cuda=False)
    t = 1.0 + r  # rank r "took" 1 + r seconds
    t_max = replicas.max_over_ranks(t, wsz, device="cpu")
    out[r] = (t_max, replicas.job_rate(w.creature_steps(), wsz, t_max), w.seed.tolist(),
              w.x.tolist())
    replicas.finish(wsz)


def test_two_gloo_ranks_shard_and_reduce():
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        port = _port()
        ps = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
        for p in ps:
            p.start()
        for p in ps:
            p.join(120)
            assert p.exitcode == 0
        (t0, rate0, seeds0, x0), (t1, rate1, seeds1, x1) = out[0], out[1]
    assert t0 == t1 == 2.0  # the slowest rank's time on every rank
    assert len(seeds0) == len(seeds1) == 32  # equal contiguous ranges of one workload
    assert not set(seeds0) & set(seeds1)  # disjoint creatures (each its own control stream)
    assert rate0 > 0


def _lonely(port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK="0", WORLD_SIZE="2",
                      LOCAL_RANK="0")
    from kraken_3_gpu_b200 import replicas
    try:
        replicas.init("gloo", 2, timeout_s=3)  # rank 1 never joins
        out["err"] = "joined"
    except Exception as e:  # noqa: BLE001
        out["err"] = type(e).__name__


def test_missing_rank_times_out_on_the_host():
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        p = ctx.Process(target=_lonely, args=(_port(), out))
        p.start()
        p.join(90)
        assert p.exitcode == 0
        assert out["err"] != "joined"


def _partition_rank(rank, world, port, out):
    """One rank of the partition / gather plumbing: its shard of one
    workload, its share of a request stream, and an ES generation whose
    evaluation is a fake of the server (fitness = a function of theta and
    the individual's index in the population)."""
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK="0")
    from kraken_3_gpu_b200 import replicas, workloads
    r, wsz, _ = replicas.dist_env()
    replicas.init("gloo", wsz, timeout_s=30)
    w = workloads.uneven(n=50, n_maps=3, seed=9, h_min=10, h_max=90)
    mine, (lo, hi) = replicas.shard(w, r, wsz, balance=True)
    requests = [k for k in range(13) if replicas.request_owner(k, wsz) == r]
    theta0 = np.arange(5, dtype=np.float32) + 1 if r == 0 else np.zeros(5, np.float32)
    seen = []

    def evaluate(theta, first, count):
        seen.append((first, count))
        return np.array([float(theta.sum()) + 1000.0 * (first + i) for i in range(count)])

    fit, theta = replicas.es_generation(evaluate, theta0, 22, r, wsz, device="cpu")
    out[r] = dict(lo=lo, hi=hi, x=mine.x.tolist(), requests=requests, fit=fit.tolist(), theta=theta.tolist(),
                  seen=seen)
    replicas.finish(wsz)


def test_two_gloo_ranks_partition_and_gather_in_global_order():
    from kraken_3_gpu_b200 import workloads
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        port = _port()
        ps = [ctx.Process(target=_partition_rank, args=(r, 2, port, out)) for r in range(2)]
        for p in ps:
            p.start()
        for p in ps:
            p.join(120)
            assert p.exitcode == 0
        a, b = dict(out[0]), dict(out[1])
    w = workloads.uneven(n=50, n_maps=3, seed=9, h_min=10, h_max=90)
    # every creature on exactly one rank, contiguous, in rank order
    assert a["lo"] == 0 and a["hi"] == b["lo"] and b["hi"] == w.n and 0 < a["hi"] < w.n
    assert np.array_equal(np.array(a["x"] + b["x"]), w.x)
    # every request on exactly one rank
    assert sorted(a["requests"] + b["requests"]) == list(range(13))
    assert not set(a["requests"]) & set(b["requests"])
    # theta from rank 0 everywhere; the gathered fitness in population order
    expect = [15.0 + 1000.0 * i for i in range(22)]
    for o in (a, b):
        assert o["theta"] == [1.0, 2.0, 3.0, 4.0, 5.0]
        assert o["fit"] == expect
    # each rank evaluated one contiguous range of whole pairs
    (fa, ca), = a["seen"]
    (fb, cb), = b["seen"]
    assert fa == 0 and fb == ca and fb % 2 == 0 and ca + cb == 22
