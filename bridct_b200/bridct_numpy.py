"""NumPy entry point with the contract of the reference's `bridct_numpy` extension.

Mirrors python/bridct_numpy.c of the reference: `Plan(height, width)` with
`forward/inverse/roundtrip(input, *, out=None)`, `close()`, and the `shape`, `route`,
`closed` properties; `core_version`.  Argument checks, their order, exception types and
messages follow python/bridct_numpy.c:84-210 so that code written against the reference
behaves the same.  The transforms run on the GPU through libbridct_b200.so
(bridct_plan_apply_batch, which streams host arrays through device staging); there is no
CPU fallback.

Drop-in use: ``import bridct_b200.bridct_numpy as bridct_numpy`` (or register it under the
name ``bridct_numpy`` in ``sys.modules``).
"""
from __future__ import annotations

import threading

import numpy as np

from . import _lib

core_version = _lib.VERSION

__all__ = ["Plan", "core_version"]


def _addr(a: np.ndarray) -> int:
    return a.__array_interface__["data"][0]


class Plan:
    """Reusable orthonormal float32 DCT plan; one plan per concurrent worker."""

    __slots__ = ("_kernel", "_height", "_width", "_initialized", "_busy", "_lock", "__weakref__")

    def __init__(self, height, width):
        if getattr(self, "_initialized", False):
            raise RuntimeError("A Plan cannot be reinitialized.")
        self._kernel = None
        self._busy = False
        self._lock = threading.Lock()
        self._initialized = False
        h, w = _as_int(height), _as_int(width)
        L = _lib.lib()
        if not L.bridct_supported(h, w):
            raise ValueError("Both dimensions must be powers of two from 8 through 1024.")
        kernel = L.bridct_plan_create(h, w)
        if not kernel:
            msg = _lib.last_error()
            if "out of memory" in msg:
                raise MemoryError(msg)
            raise RuntimeError(f"Cannot create a GPU plan: {msg}")
        self._kernel = kernel
        self._height, self._width = h, w
        self._initialized = True

    def __del__(self):
        k = getattr(self, "_kernel", None)
        if k:
            try:
                _lib.lib().bridct_plan_destroy(k)
            except Exception:  # pragma: no cover - interpreter shutdown
                pass
            self._kernel = None

    # -- properties -------------------------------------------------------------------
    @property
    def shape(self):
        return (self._height, self._width) if self._initialized else (0, 0)

    @property
    def route(self):
        if not self._kernel:
            return None
        return _lib.lib().bridct_plan_route(self._kernel).decode()

    @property
    def gpu_route(self):
        if not self._kernel:
            return None
        return _lib.lib().bridct_plan_gpu_route(self._kernel).decode()

    @property
    def closed(self):
        return not self._kernel

    # -- lifecycle --------------------------------------------------------------------
    def close(self):
        with self._lock:
            if self._busy:
                raise RuntimeError("This Plan is already initializing or executing, possibly in another thread.")
            if self._kernel:
                _lib.lib().bridct_plan_destroy(self._kernel)
            self._kernel = None

    # -- transforms -------------------------------------------------------------------
    def forward(self, *args, **kwargs):
        """forward(input, *, out=None): orthonormal 2D DCT-II over the last two axes."""
        return self._execute(args, kwargs, _lib.FORWARD)

    def inverse(self, *args, **kwargs):
        """inverse(input, *, out=None): orthonormal 2D DCT-III over the last two axes."""
        return self._execute(args, kwargs, _lib.INVERSE)

    def roundtrip(self, *args, **kwargs):
        """roundtrip(input, *, out=None): forward followed by inverse, with a materialized spectrum."""
        return self._execute(args, kwargs, _lib.ROUNDTRIP)

    def _checked(self, obj, output: bool) -> np.ndarray:
        if type(obj) is not np.ndarray:
            raise TypeError("Expected an exact NumPy ndarray; no implicit conversion is performed.")
        if obj.dtype != np.float32 or not obj.dtype.isnative:
            raise TypeError("Expected native-endian float32.")
        if (obj.ndim not in (2, 3) or obj.shape[-2] != self._height or obj.shape[-1] != self._width
                or (obj.ndim == 3 and obj.shape[0] < 1)):
            raise ValueError("Expected (height, width) or (batch, height, width), with batch >= 1.")
        if not obj.flags.c_contiguous or not obj.flags.aligned:
            raise ValueError("Expected C-contiguous, float-aligned storage.")
        if output and not obj.flags.writeable:
            raise ValueError("The output array must be writable.")
        return obj

    def _execute(self, args, kwargs, mode):
        if not self._kernel:
            raise RuntimeError("This Plan is closed or uninitialized.")
        with self._lock:
            if self._busy:
                raise RuntimeError("This Plan is executing in another thread; use one Plan per thread.")
            self._busy = True
        try:
            if len(args) != 1 or len(kwargs) > 1:
                raise TypeError("Use method(input, *, out=None).")
            out_obj = None
            if kwargs:
                (key, out_obj), = kwargs.items()
                if key != "out":
                    raise TypeError("The only accepted keyword is out.")
            x = self._checked(args[0], False)
            if out_obj is None:
                y = np.empty(x.shape, dtype=np.float32)
            else:
                y = self._checked(out_obj, True)
                if x.ndim != y.ndim or x.size != y.size:
                    raise ValueError("Input and output shapes must match exactly.")
                a, b = _addr(x), _addr(y)
                if abs(a - b) < x.nbytes:
                    raise ValueError("Input and output must not overlap.")
            batch = x.shape[0] if x.ndim == 3 else 1
            L = _lib.lib()
            if mode == _lib.ROUNDTRIP:
                # Match idct(dct(x)): the normalized spectrum is materialized in float32, in device
                # staging (bitwise the two calls; the batch crosses PCIe once each way).
                status = L.bridct_plan_roundtrip_batch(self._kernel, _addr(x), _addr(y), batch)
            else:
                status = L.bridct_plan_apply_batch(self._kernel, mode, _addr(x), _addr(y), batch)
            if status:
                raise RuntimeError(f"BRiDCT failed with status {status}.")
            return y
        finally:
            self._busy = False


def _as_int(v) -> int:
    if isinstance(v, bool) or not hasattr(v, "__index__"):
        if isinstance(v, bool):
            return int(v)
        raise TypeError("an integer is required")
    return v.__index__()
