"""Replicas over GPUs: one process per GPU, creatures sharded by rank, no
exchange on the data path (creatures are independent lanes,
src/gpu/solver.wgsl:15-18).  The only collectives are a barrier around timed
regions and the max over ranks of their times (whole-job throughput = all
ranks' creature-steps / the slowest rank's time).  Works with the nccl
backend on GPUs and with gloo on CPU."""
from __future__ import annotations

import datetime
import os

SHARD_SEED_STRIDE = 1000


def dist_env():
    """(rank, world size, local rank) from the torchrun environment."""
    return (int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)),
            int(os.environ.get("LOCAL_RANK", 0)))


def shard_seed(seed: int, rank: int) -> int:
    """Seed of a rank's shard of the synthetic workload (disjoint streams)."""
    return seed + SHARD_SEED_STRIDE * rank


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
