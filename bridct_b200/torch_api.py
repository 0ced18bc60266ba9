"""PyTorch entry point for CUDA tensors (the reference has none; it mirrors the `Plan`
semantics of the NumPy entry for device-resident data).

    y = bridct_b200.torch_api.dct2(x)          # x: (..., H, W) float32 CUDA tensor
    x = bridct_b200.torch_api.idct2(y)
    z = bridct_b200.torch_api.roundtrip2(x)

The calls are asynchronous on torch's current CUDA stream and run the plain Shao-Johnson
kernels, or a tensor-core precision form with ``form="tc_bf16x3" | "tc_tf32x3" | "tc_fp8"``.
`dct2`/`idct2` are differentiable: the transforms are orthonormal and linear, so the
gradient of the DCT-II is the DCT-III of the incoming gradient and vice versa.
"""
from __future__ import annotations

import threading
from typing import Dict, Tuple

import torch

from . import _lib

_FORMS = {"sj": _lib.FORM_SJ, "tc_bf16x3": _lib.FORM_TC_BF16X3, "tc_tf32x3": _lib.FORM_TC_TF32X3,
          "tc_fp8": _lib.FORM_TC_FP8}
_plans: Dict[Tuple[int, int, int], int] = {}
_plans_lock = threading.Lock()


def _plan(device: int, h: int, w: int) -> int:
    key = (device, h, w)
    p = _plans.get(key)
    if p:
        return p
    with _plans_lock:
        p = _plans.get(key)
        if p:
            return p
        with torch.cuda.device(device):
            p = _lib.lib().bridct_plan_create(h, w)
        if not p:
            raise RuntimeError(f"bridct_plan_create({h}, {w}) failed: {_lib.last_error()}")
        _plans[key] = p
        return p


def _check(x: torch.Tensor) -> Tuple[int, int, int]:
    if not isinstance(x, torch.Tensor):
        raise TypeError("Expected a torch.Tensor.")
    if not x.is_cuda:
        raise ValueError("Expected a CUDA tensor; use bridct_b200.bridct_numpy for host arrays.")
    if x.dtype != torch.float32:
        raise TypeError("Expected float32.")
    if x.dim() < 2:
        raise ValueError("Expected (..., height, width).")
    h, w = x.shape[-2], x.shape[-1]
    if not _lib.lib().bridct_supported(h, w):
        raise ValueError("Both dimensions must be powers of two from 8 through 1024.")
    batch = x.numel() // (h * w)
    return h, w, batch


def _strides(t: torch.Tensor):
    """(row pitch, array stride) in floats when the kernels can address t where it lies: unit
    column stride, leading dimensions that flatten to one array stride, multiples of 4 floats and a
    16-byte aligned start; else None."""
    if t.stride(-1) != 1 or t.data_ptr() % 16:
        return None
    ld = t.stride(-2) if t.shape[-2] > 1 else t.shape[-1]
    lead = [(n, s) for n, s in zip(t.shape[:-2], t.stride()[:-2]) if n != 1]
    bs = lead[-1][1] if lead else t.shape[-2] * ld
    for i in range(len(lead) - 1):
        if lead[i][1] != lead[i + 1][1] * lead[i + 1][0]:
            return None
    if ld % 4 or bs % 4 or ld < t.shape[-1]:
        return None
    return ld, bs


def apply(x: torch.Tensor, mode: int, out: torch.Tensor = None, form: str = "sj") -> torch.Tensor:
    """Transforms the last two axes of a CUDA float32 tensor (no autograd).

    The plain form reads strided views where they lie (sub-images, slices, permuted batch axes
    whose last axis has unit stride; row pitch and array stride multiples of 4 floats) and writes
    `out` likewise; other layouts, and the tensor-core forms, get a contiguous copy first."""
    h, w, batch = _check(x)
    if form not in _FORMS:
        raise ValueError(f"unknown form {form!r}; expected one of {sorted(_FORMS)}")
    if form == "sj" and batch > 0 and not x.is_contiguous():
        sx = _strides(x)
        if sx is not None:
            if out is None:
                out = torch.empty(x.shape, dtype=torch.float32, device=x.device)
            elif out.shape != x.shape or out.dtype != torch.float32 or out.device != x.device:
                raise ValueError("Input and output shapes must match exactly.")
            so = _strides(out)
            if so is not None:
                return _apply_strided(x, sx, out, so, mode, h, w, batch)
    x = x.contiguous()
    if x.data_ptr() % 16:
        x = x.clone()
    if out is None:
        out = torch.empty_like(x)
    else:
        if out.shape != x.shape or out.dtype != torch.float32 or out.device != x.device:
            raise ValueError("Input and output shapes must match exactly.")
        if not out.is_contiguous() or out.data_ptr() % 16:
            raise ValueError("Expected a contiguous, 16-byte aligned output.")
    if batch == 0:
        return out
    L = _lib.lib()
    fid = _FORMS[form]
    with torch.cuda.device(x.device):
        dev = torch.cuda.current_device()
        plan = _plan(dev, h, w)
        stream = torch.cuda.current_stream().cuda_stream
        # A tensor-core form's intermediate comes from torch's caching allocator on this stream, so
        # that calls from several streams or threads on one cached plan never share scratch.
        nbytes = L.bridct_plan_form_workspace_bytes(plan, fid, batch)
        ws = torch.empty(max(1, nbytes), dtype=torch.uint8, device=x.device) if nbytes else None
        st = L.bridct_plan_apply_form_device_ws(plan, mode, fid, x.data_ptr(), out.data_ptr(), batch,
                                                ws.data_ptr() if ws is not None else None, nbytes, stream)
    _lib.check(st, "bridct_plan_apply_form_device_ws")
    return out


def _apply_strided(x, sx, out, so, mode, h, w, batch):
    L = _lib.lib()
    with torch.cuda.device(x.device):
        plan = _plan(torch.cuda.current_device(), h, w)
        st = L.bridct_plan_apply_strided_device(plan, mode, x.data_ptr(), sx[0], sx[1], out.data_ptr(), so[0], so[1],
                                                batch, torch.cuda.current_stream().cuda_stream)
    _lib.check(st, "bridct_plan_apply_strided_device")
    return out


class _DCT2(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x, form):
        ctx.form = form
        return apply(x, _lib.FORWARD, form=form)

    @staticmethod
    def backward(ctx, g):
        return apply(g.contiguous(), _lib.INVERSE, form=ctx.form), None


class _IDCT2(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x, form):
        ctx.form = form
        return apply(x, _lib.INVERSE, form=form)

    @staticmethod
    def backward(ctx, g):
        return apply(g.contiguous(), _lib.FORWARD, form=ctx.form), None


def dct2(x: torch.Tensor, form: str = "sj") -> torch.Tensor:
    """Orthonormal 2D DCT-II over the last two axes (differentiable)."""
    return _DCT2.apply(x, form)


def idct2(x: torch.Tensor, form: str = "sj") -> torch.Tensor:
    """Orthonormal 2D DCT-III over the last two axes (differentiable)."""
    return _IDCT2.apply(x, form)


def roundtrip2(x: torch.Tensor) -> torch.Tensor:
    """Normalized round trip DCT-III(DCT-II(x)) in one pass per axis."""
    return apply(x, _lib.ROUNDTRIP)


def image_blocks8(image: torch.Tensor, mode: int = 0, quant=None, out: torch.Tensor = None) -> torch.Tensor:
    """Transforms every 8x8 block of a 2D float32 CUDA image where it lies (one launch).

    `image` may be a strided view (row stride a multiple of 4, last stride 1); `quant` is an
    optional 8x8 table of positive steps: forward returns rint(Y / Q), inverse dequantizes first,
    roundtrip quantizes and dequantizes between the two.  `out` may be `image` itself.
    """
    if not (image.is_cuda and image.dtype == torch.float32 and image.dim() == 2 and image.stride(1) == 1):
        raise ValueError("expected a 2D float32 CUDA tensor with unit column stride")
    h, w = image.shape
    if out is None:
        out = torch.empty((h, w), dtype=torch.float32, device=image.device)
    if out.shape != image.shape or out.stride(1) != 1 or out.device != image.device or out.dtype != torch.float32:
        raise ValueError("out must be a float32 tensor of the image's shape on its device with unit column stride")
    q = None
    if quant is not None:
        import numpy as np

        qa = np.ascontiguousarray(np.asarray(quant, dtype=np.float32).reshape(64))
        q = qa.ctypes.data
    with torch.cuda.device(image.device):
        st = _lib.lib().bridct_image_blocks8_device(mode, image.data_ptr(), image.stride(0), out.data_ptr(),
                                                    out.stride(0), h, w, q,
                                                    torch.cuda.current_stream().cuda_stream)
    _lib.check(st, "bridct_image_blocks8_device")
    return out


class Plan:
    """Torch counterpart of bridct_numpy.Plan for CUDA tensors of one (height, width)."""

    def __init__(self, height: int, width: int, form: str = "sj"):
        if not _lib.lib().bridct_supported(height, width):
            raise ValueError("Both dimensions must be powers of two from 8 through 1024.")
        self.shape = (height, width)
        self.form = form

    def _go(self, x, mode, out):
        if tuple(x.shape[-2:]) != self.shape:
            raise ValueError("Expected (..., height, width) matching the plan.")
        return apply(x, mode, out=out, form=self.form if mode != _lib.ROUNDTRIP else "sj")

    def forward(self, x, *, out=None):
        return self._go(x, _lib.FORWARD, out)

    def inverse(self, x, *, out=None):
        return self._go(x, _lib.INVERSE, out)

    def roundtrip(self, x, *, out=None):
        return self._go(x, _lib.ROUNDTRIP, out)
