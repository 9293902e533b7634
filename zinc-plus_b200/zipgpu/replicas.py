"""Replica execution across GPUs (one process per GPU, torch.distributed).

Zip+ commit+prove requests share nothing, so N GPUs run N replicas: each rank
takes its own share of the requests and no data moves between ranks.  The only
collectives are the barrier around a timed region and the reductions of its
timing: the job's time is the slowest rank's, and its throughput is all ranks'
units over that time.
"""
from __future__ import annotations


def shard(n: int, rank: int, world: int) -> list[int]:
    """Request indices of `rank`: round-robin, so ranks differ by at most one."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank must be in [0, world)")
    return list(range(rank, n, world))


def _reduce(x: float, op: str, dist=None, device: str = "cpu") -> float:
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(x)
    import torch

    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max" else dist.ReduceOp.SUM)
    return float(t.item())


def max_over_ranks(x: float, dist=None, device: str = "cpu") -> float:
    return _reduce(x, "max", dist, device)


def sum_over_ranks(x: float, dist=None, device: str = "cpu") -> float:
    return _reduce(x, "sum", dist, device)


def job_throughput(units: float, seconds: float, dist=None, device: str = "cpu") -> dict:
    """Whole-job throughput of a timed region: the sum of every rank's units over
    the slowest rank's time."""
    total = sum_over_ranks(units, dist, device)
    slowest = max_over_ranks(seconds, dist, device)
    return {"units": total, "seconds": slowest, "value": total / slowest if slowest > 0 else 0.0}
