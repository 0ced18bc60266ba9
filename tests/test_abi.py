"""C-ABI checks that need no GPU: the library loads, exports every declared symbol, and the
host-side validation of the reference API (argument order and status codes) holds before any
device work (tests/test_api.c:47-61,85-90 and tests/test_small_optimized.c:41-93 of the
reference)."""
import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

from bridct_b200 import _lib

ROOT = Path(__file__).resolve().parents[1]


def declared_symbols():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        for m in re.finditer(r"BRIDCT_API\s+[\w\s\*]+?\b(bridct_\w+)\s*\(", h.read_text()):
            names.add(m.group(1))
    return sorted(names)


def test_library_exports_every_declared_symbol():
    L = _lib.lib()
    names = declared_symbols()
    assert len(names) >= 13
    for n in names:
        assert hasattr(L, n), n


def test_supported_truth_table():
    L = _lib.lib()
    sizes = [8, 16, 32, 64, 128, 256, 512, 1024]
    for h in sizes:
        for w in sizes:
            assert L.bridct_supported(h, w) == 1
    for bad in [(32, 26), (-8, 16), (2048, 8), (4, 8), (8, 0), (1023, 8), (8, 1536)]:
        assert L.bridct_supported(*bad) == 0
    assert not L.bridct_plan_create(32, 26)
    assert not L.bridct_plan_create(-8, 32)
    assert not L.bridct_plan_create(2048, 8)


def test_workspace_floats_matches_reference_formula():
    L = _lib.lib()
    assert L.bridct_workspace_floats(8) == 128 and L.bridct_workspace_floats(16) == 512
    for n in (32, 64, 128, 256):
        assert L.bridct_workspace_floats(n) == 8 * n * n + 2 * 1100 * 4 + 4 * 4 * 256 + 4 * n * (4 * n + 4)
    for n in (26, -8, 0, 512, 1024):
        assert L.bridct_workspace_floats(n) == 0


def test_null_plan_handling():
    L = _lib.lib()
    assert L.bridct_plan_route(None) is None
    assert L.bridct_plan_gpu_route(None) is None
    assert L.bridct_plan_apply(None, 0, None, None) == _lib.INVALID_ARGUMENT
    L.bridct_plan_destroy(None)
    assert L.bridct_plan_apply_batch(None, 0, None, None, 1) == _lib.INVALID_ARGUMENT
    assert L.bridct_plan_apply_device(None, 0, None, None, 1, None) == _lib.INVALID_ARGUMENT


def _addr(a):
    return a.ctypes.data


def test_caller_workspace_validation_order():
    """invalid -> too small -> alignment -> overlap, with nothing written (src/bridct.c:33-45)."""
    L = _lib.lib()
    n = 8
    count = L.bridct_workspace_floats(n)
    buf = np.zeros(count + 64 + 8, np.float32)
    off = (-buf.ctypes.data // 4) % 4          # 16-byte aligned view
    ws = buf[off:off + count]
    x = np.ones(64, np.float32)
    y = np.full(64, 7.0, np.float32)
    A = L.bridct_apply
    assert A(n, 0, None, _addr(y), _addr(ws), count) == _lib.INVALID_ARGUMENT
    assert A(n, 9, _addr(x), _addr(y), _addr(ws), count) == _lib.INVALID_ARGUMENT
    assert A(26, 0, _addr(x), _addr(y), _addr(ws), count) == _lib.INVALID_ARGUMENT
    assert A(n, 0, _addr(x), _addr(y), None, count) == _lib.INVALID_ARGUMENT
    assert A(n, 0, _addr(x), _addr(y), _addr(ws), count - 1) == _lib.WORKSPACE_TOO_SMALL
    assert A(n, 0, _addr(x), _addr(y), _addr(ws) + 4, count) == _lib.BAD_ALIGNMENT
    assert A(n, 0, _addr(x), _addr(x), _addr(ws), count) == _lib.OVERLAPPING_BUFFERS
    assert A(n, 0, _addr(x), _addr(ws), _addr(ws), count) == _lib.OVERLAPPING_BUFFERS
    assert A(n, 0, _addr(ws), _addr(y), _addr(ws), count) == _lib.OVERLAPPING_BUFFERS
    assert np.all(y == 7.0)


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:  # pragma: no cover
        return False


@pytest.mark.skipif(_has_gpu(), reason="checks the no-device failure path")
def test_plan_create_fails_loudly_without_device():
    L = _lib.lib()
    assert not L.bridct_plan_create(8, 8)
    assert "CUDA" in _lib.last_error()


def test_numpy_plan_rejects_unsupported_shape_before_device_work():
    from bridct_b200.bridct_numpy import Plan
    for bad in [(32, 26), (-8, 32), (2048, 8)]:
        with pytest.raises(ValueError, match="powers of two"):
            Plan(*bad)
