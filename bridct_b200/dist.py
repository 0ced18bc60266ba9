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


def max_over_ranks(value, device=None):
    """Max over the default process group of a scalar, or elementwise of a list of scalars
    (identity without a group)."""
    import torch
    import torch.distributed as dist

    many = isinstance(value, (list, tuple))
    vals = [float(v) for v in value] if many else [float(value)]
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return vals if many else vals[0]
    t = torch.tensor(vals, dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    out = [float(v) for v in t.cpu().tolist()]
    return out if many else out[0]
