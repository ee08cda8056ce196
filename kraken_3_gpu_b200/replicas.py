"""Multi-GPU partitioning: one process per GPU, no exchange on the data path
(creatures are independent lanes, src/gpu/solver.wgsl:15-18).

  * a workload (configs of 1,024 or 16,384 creatures and up) is split into
    contiguous creature ranges, one per rank (contiguous_range / shard);
  * a stream of rollout requests goes round robin, request k to rank
    k mod world (request_owner), each rank feeding its own server;
  * an ES generation -- the reference's lockstep generation loop
    (src/sim/gputrain.js:140-150) over mirrored individuals theta +- sigma
    eps_k (src/brain/es.js:67-81) -- broadcasts theta from rank 0, lets
    every rank evaluate a contiguous range of the population's mirrored
    pairs (the server's first_individual keeps each individual's eps), and
    all-gathers the per-individual fitness in population order
    (es_generation).
Beyond those edges the only collectives are a barrier around timed regions
and the max over ranks of their times (whole-job throughput = all ranks'
creature-steps / the slowest rank's time).  Works with the nccl backend on
GPUs and with gloo on CPU.
"""
from __future__ import annotations

import datetime
import os

import numpy as np

def dist_env():
    """(rank, world size, local rank) from the torchrun environment."""
    return (int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)),
            int(os.environ.get("LOCAL_RANK", 0)))


def init(backend: str, world: int, local: int = 0, timeout_s: float = 120.0):
    """Join the process group (world > 1); a short timeout ends a stuck rank."""
    if world <= 1:
        return
    import torch
    import torch.distributed as dist
    kw = {}
    if backend == "nccl":
        kw["device_id"] = torch.device("cuda", local)
    dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s), **kw)


def barrier(world: int, cuda: bool = True):
    import torch
    if world > 1:
        torch.distributed.barrier()
    if cuda:
        torch.cuda.synchronize()


def max_over_ranks(x: float, world: int, device: str = "cuda") -> float:
    """The max of x over all ranks (every rank calls it in the same order)."""
    if world <= 1:
        return float(x)
    import torch
    t = torch.tensor([float(x)], device=device, dtype=torch.float64)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


def job_rate(units_per_rank: float, world: int, t_max_s: float) -> float:
    """Whole-job throughput: every rank's units over the slowest rank's time."""
    return world * units_per_rank / t_max_s


def finish(world: int):
    if world > 1:
        import torch
        torch.distributed.destroy_process_group()


# ---------------------------------------------------------------------------
# partitioning
# ---------------------------------------------------------------------------
def contiguous_range(n: int, rank: int, world: int, weights=None):
    """[lo, hi) of rank's contiguous share of n units.  Without weights the
    shares differ by at most one unit; with weights (one per unit, e.g.
    horizon x body cost) each boundary is the first unit where the cumulative
    weight reaches rank / world of the total.  Every unit lands on exactly one
    rank, in rank order."""
    if world <= 1:
        return 0, n
    if weights is None:
        return (n * rank) // world, (n * (rank + 1)) // world
    c = np.cumsum(np.asarray(weights, dtype=np.float64))
    total = c[-1] if n else 0.0

    def cut(r):
        if r <= 0:
            return 0
        if r >= world:
            return n
        return int(np.searchsorted(c, total * r / world, side="left")) + 1

    return min(cut(rank), n), min(cut(rank + 1), n)


def shard(w, rank: int, world: int, balance: bool = False):
    """The creatures [lo, hi) of workload w that rank runs (maps and lights
    shared); balance: split by horizon x body size instead of by count."""
    from .workloads import Workload
    weights = None
    if balance:
        weights = w.horizon.astype(np.float64) * (w.arms * (2 * w.segs + 1)).astype(np.float64)
    lo, hi = contiguous_range(w.n, rank, world, weights)
    sl = slice(lo, hi)
    return Workload(f"{w.name}[{lo}:{hi}]", w.maps, w.arms[sl], w.segs[sl], w.map_id[sl], w.x[sl], w.y[sl],
                    w.angle[sl], w.horizon[sl], w.seed[sl], w.lights), (lo, hi)


def request_owner(k: int, world: int) -> int:
    """The rank that serves request k of a stream (round robin)."""
    return k % world if world > 1 else 0


def pair_range(population: int, rank: int, world: int):
    """(first individual, individuals) of rank's contiguous share of a
    mirrored population's pairs; first is even, so each pair stays whole."""
    pairs = population // 2
    lo, hi = contiguous_range(pairs, rank, world)
    first, count = 2 * lo, 2 * (hi - lo)
    if rank == world - 1 and population % 2:
        count += 1  # an odd population's last, unpaired individual
    return first, count


def broadcast_theta(theta, world: int, device: str = "cuda"):
    """Rank 0's theta on every rank (one broadcast; a few KB)."""
    theta = np.ascontiguousarray(theta, dtype=np.float32)
    if world <= 1:
        return theta
    import torch
    t = torch.from_numpy(theta.copy()).to(device)
    torch.distributed.broadcast(t, src=0)
    return t.cpu().numpy()


def gather_fitness(local, counts, world: int, device: str = "cuda"):
    """Every rank's per-individual values (rank r holds counts[r]) in rank
    order on every rank: each piece padded to the largest, one all-gather."""
    local = np.ascontiguousarray(local, dtype=np.float64).reshape(-1)
    if world <= 1:
        return local.copy()
    import torch
    width = max(1, max(counts))
    t = torch.zeros(width, dtype=torch.float64, device=device)
    t[:local.size] = torch.from_numpy(local).to(device)
    parts = [torch.empty_like(t) for _ in range(world)]
    torch.distributed.all_gather(parts, t)
    return np.concatenate([parts[r][:counts[r]].cpu().numpy() for r in range(world)])


def es_generation(evaluate, theta, population: int, rank: int, world: int, device: str = "cuda"):
    """One ES generation over all ranks: theta from rank 0, each rank's
    contiguous range of mirrored pairs evaluated by
    evaluate(theta, first_individual, count) -> (count,) fitness, and the
    whole population's fitness gathered in individual order.  Returns
    (fitness (population,), theta)."""
    theta = broadcast_theta(theta, world, device)
    first, count = pair_range(population, rank, world)
    local = evaluate(theta, first, count) if count else np.zeros(0)
    counts = [pair_range(population, r, world)[1] for r in range(world)]
    return gather_fitness(local, counts, world, device), theta
