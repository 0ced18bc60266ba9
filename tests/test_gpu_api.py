"""Reference plan-API behaviour through the C-ABI on the GPU (the reference's
tests/test_api.c, tests/test_runner.c guard zones, tests/verify_plan.py bitwise agreement of
the plan and caller-workspace paths), with host, pinned and device pointers."""
import ctypes as C
import threading

import numpy as np
import pytest
import torch

from bridct_b200 import _lib
from oracle import oracle as O
from tests.helpers import TOL

pytestmark = pytest.mark.gpu

SHAPES12 = [(8, 8), (16, 16), (32, 32), (64, 64), (128, 128), (256, 256), (16, 32), (8, 64), (32, 16),
            (512, 512), (1024, 1024), (512, 1024)]


def addr(a):
    return a.ctypes.data


def check_shape(h, w):
    """tests/test_api.c:13-44 of the reference."""
    L = _lib.lib()
    count = h * w
    x = np.sin(np.arange(count, dtype=np.float64) * 0.017).astype(np.float32).reshape(h, w)
    saved = x.copy()
    y = np.empty_like(x)
    p = L.bridct_plan_create(h, w)
    assert p
    try:
        for mode in range(3):
            assert L.bridct_plan_apply(p, mode, addr(x), addr(y)) == 0
            assert np.array_equal(x, saved)
            assert np.isfinite(y).all()
            if mode == 2:
                assert np.abs(y - x).max() < 2e-5
            assert O.rel_max_error(y, O.fp64_apply(x, mode), x, output_scaled=True) <= TOL
        assert L.bridct_plan_apply(p, 0, addr(x), addr(x)) == _lib.OVERLAPPING_BUFFERS
        assert L.bridct_plan_apply(p, 0, addr(x), addr(x) + 4) == _lib.OVERLAPPING_BUFFERS
        assert L.bridct_plan_apply(p, -1, addr(x), addr(y)) == _lib.INVALID_ARGUMENT
        assert L.bridct_plan_apply(p, 0, None, addr(y)) == _lib.INVALID_ARGUMENT
        want = "paper8-square" if h == w and h <= 256 else "blocked-extension"
        assert L.bridct_plan_route(p).decode() == want
    finally:
        L.bridct_plan_destroy(p)


@pytest.mark.parametrize("shape", SHAPES12)
def test_reference_api_shapes(shape):
    check_shape(*shape)


def test_four_threads_independent_plans():
    errors = []

    def worker():
        try:
            for _ in range(10):
                check_shape(16, 32)
                check_shape(32, 32)
        except Exception as e:  # pragma: no cover - reported below
            errors.append(e)

    ts = [threading.Thread(target=worker) for _ in range(4)]
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    assert not errors, errors


@pytest.mark.parametrize("shape", [(8, 8), (64, 64), (16, 1024), (1024, 1024)])
def test_guard_zones_and_input_preserved(shape):
    """tests/test_runner.c:30-46: 4-float 12345.0 guards around input and output."""
    L = _lib.lib()
    h, w = shape
    n = h * w
    rng = np.random.default_rng(n)
    xin = np.full(n + 8, 12345.0, np.float32)
    yout = np.full(n + 8, 12345.0, np.float32)
    xin[4:-4] = rng.standard_normal(n)
    saved = xin.copy()
    p = L.bridct_plan_create(h, w)
    try:
        for mode in range(3):
            assert L.bridct_plan_apply(p, mode, addr(xin) + 16, addr(yout) + 16) == 0
            assert np.array_equal(xin, saved)
            assert (yout[:4] == 12345.0).all() and (yout[-4:] == 12345.0).all()
    finally:
        L.bridct_plan_destroy(p)


@pytest.mark.parametrize("shape", [(8, 8), (32, 64), (256, 256), (1024, 512)])
def test_pointer_kinds_agree_bitwise(shape):
    """Pageable, pinned, device and float-aligned (not 16-byte aligned) device pointers."""
    L = _lib.lib()
    h, w = shape
    x = np.random.default_rng(3).standard_normal((h, w)).astype(np.float32)
    p = L.bridct_plan_create(h, w)
    try:
        for mode in range(3):
            y_host = np.empty_like(x)
            assert L.bridct_plan_apply(p, mode, addr(x), addr(y_host)) == 0
            xp = torch.from_numpy(x).pin_memory()
            yp = torch.empty_like(xp).pin_memory()
            assert L.bridct_plan_apply(p, mode, xp.data_ptr(), yp.data_ptr()) == 0
            assert np.array_equal(yp.numpy(), y_host)
            xd = torch.from_numpy(x).cuda()
            yd = torch.empty_like(xd)
            assert L.bridct_plan_apply(p, mode, xd.data_ptr(), yd.data_ptr()) == 0
            assert np.array_equal(yd.cpu().numpy(), y_host)
            # float-aligned device buffers (offset by one float)
            xo = torch.zeros(h * w + 1, device="cuda")
            yo = torch.zeros(h * w + 1, device="cuda")
            xo[1:] = xd.reshape(-1)
            assert L.bridct_plan_apply(p, mode, xo.data_ptr() + 4, yo.data_ptr() + 4) == 0
            assert np.array_equal(yo[1:].cpu().numpy().reshape(h, w), y_host)
            assert yo[0].item() == 0.0
    finally:
        L.bridct_plan_destroy(p)


@pytest.mark.parametrize("n", [8, 16, 32, 64, 128, 256])
def test_caller_workspace_path_matches_plan_bitwise(n):
    """tests/verify_plan.py:38-42: bridct_apply and the plan agree bit for bit."""
    L = _lib.lib()
    count = L.bridct_workspace_floats(n)
    buf = np.zeros(count + 8, np.float32)
    off = (-buf.ctypes.data // 4) % 4
    ws = buf[off:off + count]
    x = np.random.default_rng(n).standard_normal((n, n)).astype(np.float32)
    p = L.bridct_plan_create(n, n)
    try:
        for mode in range(3):
            a = np.empty_like(x)
            b = np.empty_like(x)
            assert L.bridct_plan_apply(p, mode, addr(x), addr(a)) == 0
            assert L.bridct_apply(n, mode, addr(x), addr(b), addr(ws), count) == 0
            assert np.array_equal(a, b)
    finally:
        L.bridct_plan_destroy(p)


@pytest.mark.parametrize("shape", [(8, 8), (64, 64), (128, 1024)])
def test_batch_api_host_and_device(shape):
    L = _lib.lib()
    h, w = shape
    b = 37
    x = np.random.default_rng(5).standard_normal((b, h, w)).astype(np.float32)
    p = L.bridct_plan_create(h, w)
    try:
        for mode in range(3):
            single = np.empty_like(x)
            for i in range(b):
                assert L.bridct_plan_apply(p, mode, addr(x[i]), addr(single[i])) == 0
            yb = np.empty_like(x)
            assert L.bridct_plan_apply_batch(p, mode, addr(x), addr(yb), b) == 0
            assert np.array_equal(yb, single)
            xp = torch.from_numpy(x).pin_memory()
            yp = torch.empty_like(xp).pin_memory()
            assert L.bridct_plan_apply_batch(p, mode, xp.data_ptr(), yp.data_ptr(), b) == 0
            assert np.array_equal(yp.numpy(), single)
            xd = torch.from_numpy(x).cuda()
            yd = torch.empty_like(xd)
            assert L.bridct_plan_apply_batch(p, mode, xd.data_ptr(), yd.data_ptr(), b) == 0
            assert np.array_equal(yd.cpu().numpy(), single)
        assert L.bridct_plan_apply_batch(p, 0, addr(x), addr(x[1]), 2) == _lib.OVERLAPPING_BUFFERS
    finally:
        L.bridct_plan_destroy(p)


def test_device_api_rejects_misaligned_and_overlap_without_writing():
    L = _lib.lib()
    p = L.bridct_plan_create(8, 8)
    try:
        x = torch.randn(4, 8, 8, device="cuda")
        y = torch.full((4 * 64 + 4,), 7.0, device="cuda")
        assert L.bridct_plan_apply_device(p, 0, x.data_ptr(), y.data_ptr() + 4, 4, None) == _lib.BAD_ALIGNMENT
        assert L.bridct_plan_apply_device(p, 0, x.data_ptr(), x.data_ptr() + 64 * 4, 2, None) == \
            _lib.OVERLAPPING_BUFFERS
        assert L.bridct_plan_apply_device(p, 5, x.data_ptr(), y.data_ptr(), 4, None) == _lib.INVALID_ARGUMENT
        torch.cuda.synchronize()
        assert (y == 7.0).all()
    finally:
        L.bridct_plan_destroy(p)


def test_gpu_route_labels():
    L = _lib.lib()
    for (h, w), want in [((8, 8), "sj-tile"), ((128, 128), "sj-tile"), ((256, 256), "sj-two-pass"),
                         ((1024, 8), "sj-tile"), ((1024, 1024), "sj-two-pass")]:
        p = L.bridct_plan_create(h, w)
        assert L.bridct_plan_gpu_route(p).decode() == want
        L.bridct_plan_destroy(p)


@pytest.mark.parametrize("shape", [(262144, 8, 8), (100, 64, 64), (3, 1024, 1024), (7, 256, 512), (5, 64, 512)])
def test_back_to_back_dependent_launches(shape):
    """Each call reads the previous call's output on the same stream with no host synchronization
    in between (the plain kernels overlap their start with the previous kernel's end and wait for
    its results before their first global access): the chain forward, inverse, forward, inverse
    returns the input, and every intermediate equals the same call made alone."""
    import torch

    from bridct_b200 import torch_api

    x = torch.randn(*shape, device="cuda")
    s = torch.cuda.Stream()
    torch.cuda.synchronize()
    with torch.cuda.stream(s):
        a = torch_api.apply(x, 0)
        b = torch_api.apply(a, 1)
        c = torch_api.apply(b, 0)
        d = torch_api.apply(c, 1)
    s.synchronize()
    ref_a = torch_api.apply(x, 0)
    torch.cuda.synchronize()
    assert torch.equal(a, ref_a)
    assert torch.equal(c, torch_api.apply(b, 0))
    tol = 8e-6 * float(x.abs().max())
    assert float((d - x).abs().max()) <= tol


def test_batch_entry_points_reject_empty_null_and_bad_mode_without_writing():
    """Zero arrays, NULL buffers, a bad mode or an unknown form are INVALID_ARGUMENT on every batch
    entry point (as NULL and bad modes are on the reference's plan API, src/plan.c:129-131), and
    nothing is launched or written."""
    from bridct_b200 import torch_api

    L = _lib.lib()
    INV = _lib.INVALID_ARGUMENT
    p = torch_api._plan(torch.cuda.current_device(), 16, 32)
    x = torch.randn(2, 16, 32, device="cuda")
    y = torch.full_like(x, 7.0)
    xp, yp = x.data_ptr(), y.data_ptr()
    assert L.bridct_plan_apply_device(p, 0, xp, yp, 0, None) == INV
    assert L.bridct_plan_apply_device(p, 0, None, yp, 2, None) == INV
    assert L.bridct_plan_apply_device(p, 0, xp, None, 2, None) == INV
    for form in (_lib.FORM_TC_BF16X3, _lib.FORM_TC_TF32X3, _lib.FORM_TC_FP8):
        assert L.bridct_plan_apply_form_device(p, 0, form, xp, yp, 0, None) == INV
        assert L.bridct_plan_apply_form_device(p, 3, form, xp, yp, 2, None) == INV
        assert L.bridct_plan_apply_form_device(p, 0, form, None, yp, 2, None) == INV
        assert L.bridct_plan_form_workspace_bytes(p, form, 0) == 0
    assert L.bridct_plan_apply_form_device(p, 0, 9, xp, yp, 2, None) == INV
    assert L.bridct_plan_apply_strided_device(p, 0, xp, 32, 512, yp, 32, 512, 0, None) == INV
    assert L.bridct_plan_apply_strided_device(p, 3, xp, 32, 512, yp, 32, 512, 2, None) == INV
    xh = np.ones((2, 16, 32), np.float32)
    yh = np.full_like(xh, 7.0)
    assert L.bridct_plan_apply_batch(p, 0, xh.ctypes.data, yh.ctypes.data, 0) == INV
    assert L.bridct_plan_apply_batch(p, 3, xh.ctypes.data, yh.ctypes.data, 2) == INV
    assert L.bridct_plan_roundtrip_batch(p, xh.ctypes.data, yh.ctypes.data, 0) == INV
    assert L.bridct_plan_roundtrip_batch(p, None, yh.ctypes.data, 2) == INV
    items = (_lib.RaggedItem * 1)(_lib.RaggedItem(16, 32, 0, 0, 0))
    assert not L.bridct_ragged_create(items, 0)
    assert not L.bridct_ragged_create(None, 1)
    assert L.bridct_ragged_apply_noalloc(items, 0, xp, yp, None) == INV
    torch.cuda.synchronize()
    assert (y == 7.0).all() and (yh == 7.0).all()
