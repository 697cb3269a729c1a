"""Multi-GPU replicas: one process per GPU, each running the whole workload.

The single-GPU explicit step has no exchange, so N GPUs run N independent
replicas (weak scaling).  Timing is the max over ranks of each rank's
device time; the job's throughput counts every rank's cell updates.
These helpers are backend-agnostic (NCCL on the GPU, gloo in tests).
"""
from __future__ import annotations


def max_over_ranks(value: float, dist=None, device="cpu") -> float:
    """Maximum of a per-rank float over all ranks (the value itself when single-rank)."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_throughput(units_per_rank: float, seconds_local: float, dist=None, device="cpu") -> float:
    """Whole-job units per second: all ranks' units over the slowest rank's time."""
    world = dist.get_world_size() if (dist is not None and dist.is_initialized()) else 1
    return world * units_per_rank / max_over_ranks(seconds_local, dist, device)
