"""The multi-GPU replica plumbing (kraken_3_gpu_b200.replicas) with two gloo
ranks on the CPU: disjoint workload shards, barrier, max over ranks, the
whole-job rate, and a rank that times out instead of hanging."""
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
    w = workloads.uneven(n=32, n_maps=2, seed=replicas.shard_seed(2, r), h_min=10, h_max=20)
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
    assert not set(seeds0) & set(seeds1)  # disjoint control streams
    assert not np.allclose(x0, x1)  # different spawn points
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
