"""CPU oracle for the BRiDCT hot path: TEST INFRASTRUCTURE ONLY.

Three checkers, used by tests/, __graft_entry__.smoke() and bench.py's CPU legs, never by
the product path:

* ``fp64_apply`` - the mathematical contract in float64 (docs/API.md:7-13): FORWARD = Q_h X Q_w^T,
  INVERSE = Q_h^T X Q_w, ROUNDTRIP = X, with the orthonormal DCT-II matrix of
  dataset/corpus.py:10-12.
* ``sj_apply`` - the C restatement of the reference's Shao-Johnson route (sj_oracle.c), float32.
* ``ref_apply`` / ``ref_bench`` - the reference library itself, compiled from its own sources
  into oracle/_ref by oracle/Makefile (only where those files were built).
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path
from typing import Optional

import numpy as np

HERE = Path(__file__).resolve().parent
_FP = C.POINTER(C.c_float)
_sj = None
_ref = None
_bench = None


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(_FP)


def _load_sj():
    global _sj
    if _sj is None:
        lib = C.CDLL(str(HERE / "liboracle_sj.so"))
        lib.oracle_sj_scale.restype = C.c_double
        lib.oracle_sj_scale.argtypes = [C.c_int, C.c_int]
        lib.oracle_apply_batch.restype = C.c_int
        lib.oracle_apply_batch.argtypes = [C.c_int, C.c_int, C.c_int, C.c_size_t, _FP, _FP]
        lib.oracle_core_f.argtypes = [C.c_int, _FP, C.c_ssize_t, _FP, C.c_ssize_t]
        lib.oracle_core_t.argtypes = [C.c_int, _FP, C.c_ssize_t, _FP, C.c_ssize_t]
        lib.oracle_plan_tables.argtypes = [C.c_int, C.c_int, _FP, _FP]
        _sj = lib
    return _sj


def ref_available() -> bool:
    return (HERE / "_ref" / "libbridct_ref.so").exists()


def _load_ref():
    global _ref
    if _ref is None:
        lib = C.CDLL(str(HERE / "_ref" / "libbridct_ref.so"))
        lib.bridct_plan_create.restype = C.c_void_p
        lib.bridct_plan_create.argtypes = [C.c_int, C.c_int]
        lib.bridct_plan_destroy.argtypes = [C.c_void_p]
        lib.bridct_plan_apply.restype = C.c_int
        lib.bridct_plan_apply.argtypes = [C.c_void_p, C.c_int, _FP, _FP]
        lib.bridct_plan_route.restype = C.c_char_p
        lib.bridct_plan_route.argtypes = [C.c_void_p]
        _ref = lib
    return _ref


def _as_batch(x: np.ndarray) -> np.ndarray:
    x = np.ascontiguousarray(x, dtype=np.float32)
    return x[None] if x.ndim == 2 else x


def q_matrix(n: int) -> np.ndarray:
    """Orthonormal DCT-II matrix Q_n[k, j] = sqrt((k?2:1)/n) cos(pi k (j+1/2)/n)."""
    k = np.arange(n, dtype=np.float64)
    return np.cos(np.pi * k[:, None] * (k[None, :] + 0.5) / n) * np.sqrt(np.where(k == 0, 1.0, 2.0) / n)[:, None]


def fp64_apply(x: np.ndarray, mode: int) -> np.ndarray:
    """Float64 result of the contract for (H, W) or (B, H, W) input."""
    xd = np.asarray(x, dtype=np.float64)
    qh, qw = q_matrix(xd.shape[-2]), q_matrix(xd.shape[-1])
    if mode == 0:
        return qh @ xd @ qw.T
    if mode == 1:
        return qh.T @ xd @ qw
    return xd.copy()


def sj_apply(x: np.ndarray, mode: int) -> np.ndarray:
    """Float32 Shao-Johnson restatement (sj_oracle.c) on (H, W) or (B, H, W) input."""
    xb = _as_batch(x)
    y = np.empty_like(xb)
    rc = _load_sj().oracle_apply_batch(xb.shape[1], xb.shape[2], mode, xb.shape[0], _ptr(xb), _ptr(y))
    if rc:
        raise ValueError(f"oracle rejected shape {xb.shape[1:]} / mode {mode}")
    return y.reshape(np.shape(x))


def sj_scale(n: int, k: int) -> float:
    return _load_sj().oracle_sj_scale(n, k)


def sj_core(x1d: np.ndarray, transpose: bool = False) -> np.ndarray:
    x = np.ascontiguousarray(x1d, dtype=np.float32)
    y = np.empty_like(x)
    (_load_sj().oracle_core_t if transpose else _load_sj().oracle_core_f)(x.size, _ptr(x), 1, _ptr(y), 1)
    return y


def ref_apply(x: np.ndarray, mode: int) -> np.ndarray:
    """The reference library itself (oracle/_ref), one bridct_plan_apply per array."""
    lib = _load_ref()
    xb = _as_batch(x)
    y = np.empty_like(xb)
    plan = lib.bridct_plan_create(xb.shape[1], xb.shape[2])
    if not plan:
        raise ValueError("reference rejected the shape")
    try:
        for i in range(xb.shape[0]):
            rc = lib.bridct_plan_apply(plan, mode, _ptr(xb[i]), _ptr(y[i]))
            if rc:
                raise RuntimeError(f"reference status {rc}")
    finally:
        lib.bridct_plan_destroy(plan)
    return y.reshape(np.shape(x))


def bench_available() -> bool:
    return (HERE / "_ref" / "libref_bench.so").exists()


def ref_bench(hs, ws, modes, offsets, x: np.ndarray, y: np.ndarray, threads: int, repeats: int) -> float:
    """Times the reference library on the host cores; returns seconds for `repeats` passes."""
    global _bench
    if _bench is None:
        lib = C.CDLL(str(HERE / "_ref" / "libref_bench.so"))
        lib.ref_bench_run.restype = C.c_double
        lib.ref_bench_run.argtypes = [C.c_size_t, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int),
                                      C.POINTER(C.c_size_t), _FP, _FP, C.c_int, C.c_size_t]
        _bench = lib
    hs = np.ascontiguousarray(hs, dtype=np.int32)
    ws = np.ascontiguousarray(ws, dtype=np.int32)
    modes = np.ascontiguousarray(modes, dtype=np.int32)
    offsets = np.ascontiguousarray(offsets, dtype=np.uint64)
    ip = C.POINTER(C.c_int)
    t = _bench.ref_bench_run(len(hs), hs.ctypes.data_as(ip), ws.ctypes.data_as(ip), modes.ctypes.data_as(ip),
                             offsets.ctypes.data_as(C.POINTER(C.c_size_t)), _ptr(x), _ptr(y), threads, repeats)
    if t < 0:
        raise RuntimeError(f"reference bench failed ({t})")
    return t


def host_threads() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:  # pragma: no cover
        return os.cpu_count() or 1


def rel_max_error(y: np.ndarray, ref: np.ndarray, x: np.ndarray, output_scaled: bool = False) -> float:
    """max|y - ref| / max|x| per array, worst array (the bound's metric).

    With output_scaled, the denominator is max(max|x|, max|ref|) per array.
    """
    y = np.asarray(y, dtype=np.float64)
    ref = np.asarray(ref, dtype=np.float64)
    x = np.asarray(x, dtype=np.float64)
    if y.ndim == 2:
        y, ref, x = y[None], ref[None], x[None]
    num = np.abs(y - ref).reshape(len(y), -1).max(axis=1)
    den = np.abs(x).reshape(len(x), -1).max(axis=1)
    if output_scaled:
        den = np.maximum(den, np.abs(ref).reshape(len(ref), -1).max(axis=1))
    den = np.where(den == 0, 1.0, den)
    return float((num / den).max())


def rel_rms_error(y: np.ndarray, ref: np.ndarray, x: np.ndarray) -> float:
    y = np.asarray(y, dtype=np.float64)
    ref = np.asarray(ref, dtype=np.float64)
    x = np.asarray(x, dtype=np.float64)
    if y.ndim == 2:
        y, ref, x = y[None], ref[None], x[None]
    num = np.sqrt(((y - ref) ** 2).reshape(len(y), -1).mean(axis=1))
    den = np.abs(x).reshape(len(x), -1).max(axis=1)
    den = np.where(den == 0, 1.0, den)
    return float((num / den).max())
