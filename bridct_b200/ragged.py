"""Batching form: thousands of arrays of mixed shapes and directions in one persistent launch.

    batch = RaggedBatch([(h, w, mode), ...])      # offsets packed, 16-byte aligned
    y = batch.apply(x)                             # x: flat float32 CUDA tensor of batch.span floats
    batch.unpack(y)                                # list of (h, w) tensors

The work queue (column strips, row blocks and whole small arrays) is built once on the host;
`apply` is one counter reset plus one kernel on torch's current stream, so it can be captured in
a CUDA graph.  A schedule can instead give shape classes their own fixed-shape launches, forked
onto side streams inside the same call (still capturable).  `apply_loop` runs the same batch as one
plain-form launch per array, the comparison baseline.  The unit geometry and the per-class
schedule come from the autotuner (bridct_b200.autotune).
"""
from __future__ import annotations

from typing import Iterable, List, Optional, Sequence, Tuple

import numpy as np

from . import _lib


def pack_offsets(shapes: Sequence[Tuple[int, int]]) -> Tuple[np.ndarray, int]:
    """Offsets (floats, multiples of 4) for arrays packed back to back; returns (offsets, span)."""
    offs = np.zeros(len(shapes), dtype=np.int64)
    pos = 0
    for i, (h, w) in enumerate(shapes):
        offs[i] = pos
        pos += h * w            # h*w is a multiple of 64, so every offset stays 16-byte aligned
    return offs, pos


SCHEDULES = {"queue": 0, "launch": 1, "launch_small": 2, "merged": 3}


def two_pass(h: int, w: int, mode: int) -> bool:
    """Whether the plain form runs (h, w, mode) as a column pass then a row pass (the classes that
    may take the "merged" schedule): every shape above 16384 floats except whole 32768-float
    arrays in the modes where one tile measured faster (plain_launch.cuh, whole_array_route)."""
    whole = h * w == 32768 and (mode == 1 or h in (1024, 64) or (h == 32 and mode == 0))
    return h * w > 16384 and not whole


class RaggedBatch:
    def __init__(self, items: Iterable[Tuple[int, int, int]], offsets: Optional[Sequence[int]] = None,
                 tuning: Optional[dict] = None, schedule: Optional[dict] = None):
        items = list(items)
        shapes = [(h, w) for h, w, _ in items]
        if offsets is None:
            offsets, span = pack_offsets(shapes)
        else:
            offsets = np.asarray(offsets, dtype=np.int64)
            span = int(max(o + h * w for o, (h, w) in zip(offsets, shapes)))
        self.items = items
        self.offsets = offsets
        self.span = int(span)
        arr = (_lib.RaggedItem * len(items))()
        for i, ((h, w, m), o) in enumerate(zip(items, offsets)):
            arr[i] = _lib.RaggedItem(h, w, m, 0, int(o))
        L = _lib.lib()
        if tuning is None:
            self._h = L.bridct_ragged_create(arr, len(items))
        else:
            t = _lib.RaggedTuning()
            L.bridct_ragged_default_tuning(t)
            for k, v in tuning.items():
                setattr(t, k, int(v))
            self._h = L.bridct_ragged_create_tuned(arr, len(items), t)
        if not self._h:
            raise ValueError(f"bridct_ragged_create failed: {_lib.last_error()}")
        if schedule:
            self.set_schedule(schedule)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            try:
                _lib.lib().bridct_ragged_destroy(h)
            except Exception:  # pragma: no cover - interpreter shutdown
                pass
            self._h = None

    @property
    def units(self) -> int:
        return int(_lib.lib().bridct_ragged_units(self._h))

    def launch_count(self) -> int:
        """Kernel launches of one apply with the current schedule."""
        return int(_lib.lib().bridct_ragged_launch_count(self._h))

    def classes(self) -> List[dict]:
        """Shape classes, largest first: {"key": "HxW/mode", "h", "w", "mode", "arrays", "schedule"}."""
        import ctypes as C

        L = _lib.lib()
        out = []
        for i in range(int(L.bridct_ragged_class_count(self._h))):
            h, w, m, sch = C.c_int(), C.c_int(), C.c_int(), C.c_int()
            n = C.c_size_t()
            _lib.check(L.bridct_ragged_class_info(self._h, i, h, w, m, n, sch), "bridct_ragged_class_info")
            out.append({"key": f"{h.value}x{w.value}/{m.value}", "h": h.value, "w": w.value, "mode": m.value,
                        "arrays": int(n.value), "schedule": sch.value})
        return out

    def set_schedule(self, schedule: dict) -> None:
        """schedule = {"classes": {"HxW/mode": "queue"|"launch"|"launch_small"}, "streams": n};
        classes not named keep the queue."""
        import ctypes as C

        names = schedule.get("classes", {})
        cls = self.classes()
        arr = (C.c_int * max(1, len(cls)))()
        for i, c in enumerate(cls):
            v = names.get(c["key"], "queue")
            arr[i] = SCHEDULES[v] if isinstance(v, str) else int(v)
        _lib.check(_lib.lib().bridct_ragged_set_schedule(self._h, arr, len(cls), int(schedule.get("streams", 4))),
                   "bridct_ragged_set_schedule")

    def apply_class(self, index: int, schedule: str, x, y, stream=None):
        """One class alone as its own launch (for measurement)."""
        import torch

        s = torch.cuda.current_stream(x.device).cuda_stream if stream is None else stream
        _lib.check(_lib.lib().bridct_ragged_apply_class_device(self._h, index, SCHEDULES[schedule], x.data_ptr(),
                                                               y.data_ptr(), s), "ragged class apply")
        return y

    def _go(self, fn, x, y, stream):
        import torch

        if y is None:
            y = torch.empty_like(x)
        if x.numel() < self.span or y.numel() < self.span or x.dtype != torch.float32 or not x.is_cuda:
            raise ValueError("expected float32 CUDA tensors holding the packed batch")
        s = torch.cuda.current_stream(x.device).cuda_stream if stream is None else stream
        _lib.check(fn(self._h, x.data_ptr(), y.data_ptr(), s), "ragged apply")
        return y

    def apply(self, x, y=None, stream=None):
        """The whole batch: the queued classes in one persistent launch, the others as their own
        launches on forked side streams (asynchronous on the current stream)."""
        return self._go(_lib.lib().bridct_ragged_apply_device, x, y, stream)

    def apply_loop(self, x, y=None, stream=None):
        """One plain-form launch per array (baseline)."""
        return self._go(_lib.lib().bridct_ragged_apply_loop_device, x, y, stream)

    def timed_out(self) -> bool:
        return _lib.lib().bridct_ragged_timeout_flag(self._h) != 0

    def unpack(self, flat) -> List:
        return [flat[o:o + h * w].view(h, w) for (h, w, _), o in zip(self.items, self.offsets)]
