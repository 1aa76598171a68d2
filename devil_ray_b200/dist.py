"""One process per GPU for the batched workloads: the queries (or rays) are
sharded across ranks and every rank locates its own share against its own
replica of the mesh and BVH, so the data path has no collective.  The only
exchanges are the bench's: a barrier around each timed region, the maximum
of the ranks' elapsed times and the sum of their located counts.  These
helpers work with NCCL on GPUs and with gloo on CPUs (the tests run two gloo
ranks on the host)."""
from __future__ import annotations

import os
from datetime import timedelta

import torch


def dist_info():
    """(rank, world size, local rank) from the torchrun environment."""
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def init(backend: str = "nccl", timeout_s: float = 120.0):
    """The default process group when there is more than one rank, else None.
    A short timeout makes a rank that never arrives end the others' next
    collective with an error instead of a hang."""
    _, world, _ = dist_info()
    if world <= 1:
        return None
    import torch.distributed as dist
    dist.init_process_group(backend, timeout=timedelta(seconds=timeout_s))
    return dist


def shard_seed(rank: int, base: int = 1000) -> int:
    """Seed of rank's share of the synthetic queries (each rank its own)."""
    return base + rank


def _reduce(pg, value, op, dtype, device):
    if pg is None:
        return value
    t = torch.tensor([value], dtype=dtype, device=device)
    pg.all_reduce(t, op=op)
    return t.item()


def max_over_ranks(pg, value: float, device="cpu") -> float:
    """The slowest rank's time (every rank gets it)."""
    if pg is None:
        return float(value)
    return float(_reduce(pg, float(value), pg.ReduceOp.MAX, torch.float64, device))


def sum_over_ranks(pg, value: int, device="cpu") -> int:
    """Whole-job total of a per-rank count (every rank gets it)."""
    if pg is None:
        return int(value)
    return int(_reduce(pg, int(value), pg.ReduceOp.SUM, torch.int64, device))


def job_rate(pg, units: int, ms: float, device="cpu") -> float:
    """Units per second of the whole job: all ranks' units over the slowest
    rank's time (the rule every throughput in the bench follows)."""
    total = sum_over_ranks(pg, units, device)
    slowest = max_over_ranks(pg, ms, device)
    return total / (slowest * 1e-3)
