"""Multi-GPU plumbing for batches of independent arrays.

Every array is an independent unit, so a batch shards across ranks with no exchange step: each
rank transforms its own slice on its own GPU and no collective touches the data.  The only
collective is the timing reduction (max over ranks of a device-measured duration).
"""
from __future__ import annotations

from typing import Tuple


def shard_range(batch: int, rank: int, world: int) -> Tuple[int, int]:
    """(first, count) of rank's contiguous slice of `batch` arrays; slices differ by <= 1."""
    if world < 1 or not 0 <= rank < world or batch < 0:
        raise ValueError("invalid rank/world/batch")
    base, extra = divmod(batch, world)
    first = rank * base + min(rank, extra)
    return first, base + (1 if rank < extra else 0)


def max_over_ranks(value: float, device=None) -> float:
    """Max of a scalar over the default process group (identity without one)."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
