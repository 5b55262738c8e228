"""Process-per-GPU plumbing for the multi-GPU runs (torch.distributed).

Frames and BA windows are independent, so N GPUs run N shards with no collective on the data path; the only
exchanges are the timing reduction (the slowest rank defines the step time) and, if a caller wants the results on
one rank, a gather of fixed-size records.
"""
from __future__ import annotations

import os


def env():
    """(world_size, rank, local_rank) from the torchrun environment (1, 0, 0 without it)."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def shard(n, rank, world):
    """Contiguous share [a, b) of n units for `rank` of `world` (sizes differ by at most one)."""
    base, extra = divmod(int(n), int(world))
    a = rank * base + min(rank, extra)
    return a, a + base + (1 if rank < extra else 0)


def max_over_ranks(value, device=None):
    """The maximum of a float over all ranks (identity without an initialised process group)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value, device=None):
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())
