"""Multi-rank helpers of the benchmark (one process per GPU, weak scaling).

The path shards by columns with no data exchange: every rank owns a full,
independently seeded domain, and the whole-job throughput is all ranks'
cells over the slowest rank's device time.  These helpers are the only
collective steps of a multi-rank run (all ranks call them in the same
order); they work with any torch.distributed backend (NCCL on GPUs, gloo on
CPU for the tests).
"""
from __future__ import annotations


def rank_seed(base: int, rank: int) -> int:
    """Seed of rank `rank`'s domain."""
    return base + rank


def max_over_ranks(x: float, dist=None, device: str = "cuda") -> float:
    """Max of a per-rank scalar (a device time) over all ranks."""
    if dist is None:
        return float(x)
    import torch

    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def weak_scaling_value(cells_per_rank: int, steps: int, world: int, ms_max: float) -> float:
    """Whole-job cells/s: every rank's cells over the slowest rank's time."""
    return cells_per_rank * steps * world / (ms_max / 1e3)
