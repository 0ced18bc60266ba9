"""Multi-GPU plumbing for batches of independent arrays.

Every array is an independent unit, so a batch shards across ranks (or across the devices of one
process) with no exchange step: each shard is transformed on its own GPU and no collective touches
the data.  The only collective in a timed run is the timing reduction (max over ranks of a
device-measured duration).

    first, count = shard_range(batch, rank, world)     # this rank's contiguous slice
    mine, first = shard(x, rank, world)                 # the slice itself (a view)
    y = apply_sharded(x, mode, devices=[0, 1, 2, 3])    # one process driving several GPUs
    full = gather_shards(y_mine, first, batch)          # tests / callers that want one array back

A ragged batch (arrays of mixed shapes packed back to back) shards by elements instead of by
arrays, so that ranks get equal work whatever the mix:

    first, count = ragged_shard_range([h * w for h, w, _ in items], rank, world)
    my_items, x_mine, first = ragged_shard(items, x_packed, rank, world)   # a slice of the buffer
    y = apply_ragged_sharded(items, x_packed, devices=[0, 1])            # one process, two GPUs
"""
from __future__ import annotations

from typing import Callable, List, Optional, Sequence, Tuple


def shard_range(batch: int, rank: int, world: int) -> Tuple[int, int]:
    """(first, count) of rank's contiguous slice of `batch` arrays; slices differ by <= 1."""
    if world < 1 or not 0 <= rank < world or batch < 0:
        raise ValueError("invalid rank/world/batch")
    base, extra = divmod(batch, world)
    first = rank * base + min(rank, extra)
    return first, base + (1 if rank < extra else 0)


def ragged_shard_range(sizes: Sequence[int], rank: int, world: int) -> Tuple[int, int]:
    """(first, count) of rank's contiguous run of a ragged batch's arrays, balanced by elements.

    sizes[i] is array i's element count (h * w).  With the arrays packed back to back in T
    elements, rank r takes the arrays whose first element lies in [r T / world, (r + 1) T / world):
    every rank's share is within one array of T / world elements, and its arrays are one
    contiguous slice of the packed buffer (no gather)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("invalid rank/world")
    if any(int(s) < 0 for s in sizes):
        raise ValueError("negative array size")
    total = sum(int(s) for s in sizes)
    first = count = 0
    pos = 0
    for i, s in enumerate(sizes):
        owner = pos * world // total if total else 0
        if owner < rank:
            first = i + 1
        elif owner == rank:
            count += 1
        pos += int(s)
    return first, count


def ragged_shard(items: Sequence[Tuple[int, int, int]], x, rank: int, world: int):
    """Rank's share of a ragged batch packed back to back in x (a flat numpy array or tensor):
    (its items, the slice of x that holds them, index of its first item).  The slice is a view,
    itself packed back to back, so it is the input of a RaggedBatch of those items."""
    sizes = [h * w for h, w, _ in items]
    first, count = ragged_shard_range(sizes, rank, world)
    start = sum(sizes[:first])
    end = start + sum(sizes[first:first + count])
    return list(items[first:first + count]), x[start:end], first


def apply_ragged_sharded(items: Sequence[Tuple[int, int, int]], x, devices: Optional[Sequence[int]] = None,
                         transform: Optional[Callable] = None):
    """Transforms a ragged batch packed back to back in x (a flat float32 tensor or numpy array)
    split over several GPUs of this process by elements (ragged_shard): share i goes to devices[i]
    as its own RaggedBatch on that device's current stream, and the results come back in order,
    packed like x (a tensor on x's device, or a numpy array).  No collective is involved.

    `transform(items, piece, device)` replaces the per-device transform."""
    import numpy as np

    if devices is None:
        import torch

        devices = list(range(torch.cuda.device_count()))
    if not devices:
        raise ValueError("apply_ragged_sharded needs at least one device")
    if transform is None:
        transform = _ragged_device_transform
    world = len(devices)
    outs: List[Tuple[int, object]] = []
    for r, dev in enumerate(devices):
        mine, piece, first = ragged_shard(items, x, r, world)
        if mine:
            outs.append((first, mine, transform(mine, piece, dev)))
    pos = 0
    for first, mine, y in outs:                     # the shares tile the batch in order
        if first != pos:
            raise ValueError(f"ragged shares do not tile the batch: expected item {pos}, got {first}")
        pos += len(mine)
    if pos != len(items):
        raise ValueError(f"ragged shares cover {pos} of {len(items)} arrays")
    pieces = [y for _, _, y in outs]
    if isinstance(x, np.ndarray):
        return np.concatenate([np.asarray(p.cpu() if hasattr(p, "cpu") else p) for p in pieces]) if pieces \
            else np.zeros(0, np.float32)
    import torch

    return torch.cat([p.to(x.device) for p in pieces]) if pieces else x.new_empty(0)


def _ragged_device_transform(items, piece, dev):
    import numpy as np
    import torch

    from .ragged import RaggedBatch

    t = torch.from_numpy(np.ascontiguousarray(piece)) if isinstance(piece, np.ndarray) else piece
    with torch.cuda.device(dev):
        return RaggedBatch(items).apply(t.to(f"cuda:{dev}", non_blocking=True).contiguous())


def shard(x, rank: int, world: int):
    """Rank's contiguous slice of the arrays in x (leading axis) and its first index."""
    first, count = shard_range(int(x.shape[0]), rank, world)
    return x[first:first + count], first


def stitch(parts: Sequence[Tuple[int, object]], batch: int):
    """Concatenates (first, shard) pieces in order after checking that they tile [0, batch)."""
    import numpy as np

    parts = sorted(parts, key=lambda p: p[0])
    pos = 0
    for first, piece in parts:
        if first != pos:
            raise ValueError(f"shards do not tile the batch: expected first {pos}, got {first}")
        pos += int(piece.shape[0])
    if pos != batch:
        raise ValueError(f"shards cover {pos} of {batch} arrays")
    pieces = [p for _, p in parts]
    if pieces and hasattr(pieces[0], "cpu"):
        import torch

        return torch.cat([p.cpu() for p in pieces])
    return np.concatenate(pieces) if pieces else np.empty((0,))


def apply_sharded(x, mode: int, devices: Optional[Sequence[int]] = None, form: str = "sj",
                  transform: Optional[Callable] = None):
    """Transforms a batch (numpy array or tensor, (B, h, w)) split over several GPUs of this
    process: shard i goes to devices[i], each device runs its shard on its own current stream with
    its own cached plan, and the results come back stitched in order (a tensor on the input's
    device for tensor input, a numpy array for numpy input).  No collective is involved.

    `transform(piece, mode, device)` replaces the per-device transform (the default moves the
    shard to the device and runs bridct_b200.torch_api.apply)."""
    import numpy as np

    if devices is None:
        import torch

        devices = list(range(torch.cuda.device_count()))
    if not devices:
        raise ValueError("apply_sharded needs at least one device")
    if transform is None:
        transform = _device_transform(form)
    world = len(devices)
    outs: List[Tuple[int, object]] = []
    for r, dev in enumerate(devices):
        piece, first = shard(x, r, world)
        if int(piece.shape[0]):
            outs.append((first, transform(piece, mode, dev)))
    full = stitch(outs, int(x.shape[0]))
    if isinstance(x, np.ndarray):
        return full.numpy() if hasattr(full, "numpy") else full
    return full.to(x.device) if hasattr(x, "device") else full


def _device_transform(form: str):
    def run(piece, mode, dev):
        import numpy as np
        import torch

        from . import torch_api

        t = torch.from_numpy(np.ascontiguousarray(piece)) if isinstance(piece, np.ndarray) else piece
        with torch.cuda.device(dev):
            y = torch_api.apply(t.to(f"cuda:{dev}", non_blocking=True), mode, form=form)
        return y

    return run


def gather_shards(local, first: int, batch: int):
    """Rank 0 receives every rank's (first, shard) over the default process group and returns the
    stitched batch; other ranks return None.  For checking and collecting results, not for the
    timed data path."""
    import torch.distributed as dist

    world = dist.get_world_size()
    items = [None] * world
    dist.all_gather_object(items, (first, local))
    if dist.get_rank() != 0:
        return None
    return stitch(items, batch)


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
