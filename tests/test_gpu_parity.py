"""Parity of the CUDA plain (Shao-Johnson FP32) path with the oracle and the reference.

Every comparison is max|y - ref| / max(max|x|, max|ref|) per array <= 2e-6 (TOL), plus the
reference's Frobenius gate 2e-5 where it applies.  References: the float64 contract
(oracle.fp64_apply), the C restatement of the SJ route (oracle.sj_apply) and the reference
library's own outputs stored in tests/golden.
"""
import numpy as np
import pytest
import torch

from bridct_b200 import _lib, torch_api
from oracle import oracle as O
from tests.helpers import FROB, SIZES, TOL, corpus_files, frob_rel, golden, verify_families, verify_files

pytestmark = pytest.mark.gpu


def gpu(x: np.ndarray, mode: int) -> np.ndarray:
    t = torch.from_numpy(np.ascontiguousarray(x, dtype=np.float32)).cuda()
    y = torch_api.apply(t, mode)
    torch.cuda.synchronize()
    return y.cpu().numpy()


def err(y, ref, x):
    return O.rel_max_error(y, ref, x, output_scaled=True)


@pytest.mark.parametrize("h", SIZES)
def test_all_shapes_all_modes_vs_fp64_and_oracle(h):
    rng = np.random.default_rng(1000 + h)
    for w in SIZES:
        batch = max(1, min(6, 65536 // (h * w)))
        x = rng.uniform(-1, 1, (batch, h, w)).astype(np.float32)
        for m in range(3):
            y = gpu(x, m)
            assert np.isfinite(y).all()
            e64 = err(y, O.fp64_apply(x, m), x)
            esj = err(y, O.sj_apply(x, m), x)
            assert e64 <= TOL, (h, w, m, e64)
            assert esj <= TOL, (h, w, m, esj)


@pytest.mark.parametrize("path", corpus_files(), ids=lambda p: p.stem)
def test_reference_corpus(path):
    g = golden(path.name)
    x, core = g["x"], g["domain"] == "core"
    for m in range(3):
        y = gpu(x, m)
        assert err(y[core], g[f"y{m}"][core], x[core]) <= TOL
        exact = O.fp64_apply(x, m)
        for i in np.where(core)[0]:
            assert frob_rel(y[i], exact[i], x[i]) < FROB
        # boundary diagnostics: wherever the reference is finite, so are we
        fin = np.isfinite(g[f"y{m}"]).reshape(len(x), -1).all(axis=1)
        assert np.isfinite(y[fin]).all()


@pytest.mark.parametrize("path", verify_files(), ids=lambda p: p.stem)
def test_reference_verify_families(path):
    g = golden(path.name)
    x = g["x"]
    for m in range(3):
        y = gpu(x, m)
        assert err(y, g[f"y{m}"], x) <= TOL
        assert (y[0] == 0).all()                       # zero in, zero out
        for i in range(len(x)):
            assert frob_rel(y[i], O.fp64_apply(x[i], m), x[i]) < FROB


@pytest.mark.parametrize("h", [128, 256, 512, 1024])
def test_verify_families_large_shapes(h):
    """The reference's six families (tests/verify_plan.py:21-28) on shapes above 64."""
    rng = np.random.default_rng(7 + h)
    for w in (8, 128, 1024):
        x = verify_families(h, w, rng)
        for m in range(3):
            y = gpu(x, m)
            assert err(y, O.fp64_apply(x, m), x) <= TOL, (h, w, m)


def test_reference_config_samples():
    g = golden("configs.npz")
    for key in ("c1", "c2", "c3", "c5"):
        x = g[f"{key}_x"]
        for m in range(3):
            assert err(gpu(x, m), g[f"{key}_y{m}"], x) <= TOL, key


@pytest.mark.parametrize("shape,batches", [((8, 8), (1, 127, 129, 300)), ((16, 32), (1, 15, 17)),
                                           ((64, 64), (1, 3)), ((8, 1024), (1, 2, 3)),
                                           ((256, 256), (1, 3)), ((1024, 1024), (1, 2))])
def test_batch_tails_and_guards(shape, batches):
    """Partial tiles and chunk tails: every array correct, nothing written past the batch."""
    h, w = shape
    rng = np.random.default_rng(h * w)
    plan = torch_api._plan(torch.cuda.current_device(), h, w)
    for b in batches:
        x = torch.from_numpy(rng.uniform(-1, 1, (b + 1, h, w)).astype(np.float32)).cuda()
        y = torch.full_like(x, 12345.0)
        st = _lib.lib().bridct_plan_apply_device(plan, 0, x.data_ptr(), y.data_ptr(), b, None)
        assert st == 0
        torch.cuda.synchronize()
        yn = y.cpu().numpy()
        assert (yn[b] == 12345.0).all()
        xn = x.cpu().numpy()[:b]
        assert err(yn[:b], O.fp64_apply(xn, 0), xn) <= TOL


def test_config2_full_blocks():
    """262,144 independent 8x8 blocks of a 4096x4096 image (integers 0..255 minus 128)."""
    img = (np.random.default_rng(1).integers(0, 256, (4096, 4096)) - 128).astype(np.float32)
    blocks = img.reshape(512, 8, 512, 8).transpose(0, 2, 1, 3).reshape(-1, 8, 8).copy()
    y = gpu(blocks, 0)
    q = O.q_matrix(8)
    exact = np.einsum("ij,bjk,lk->bil", q, blocks.astype(np.float64), q)
    assert err(y, exact, blocks) <= TOL
    assert O.rel_max_error(y, exact, blocks) <= TOL      # literal bound holds here too
    sub = slice(0, 4096)
    assert err(y[sub], O.sj_apply(blocks[sub], 0), blocks[sub]) <= TOL
    rt = gpu(blocks, 2)
    assert O.rel_max_error(rt, blocks, blocks) <= TOL


def test_config1_full():
    x = np.random.default_rng(0).uniform(-1, 1, (1024, 64, 64)).astype(np.float32)
    for m in range(3):
        assert err(gpu(x, m), O.fp64_apply(x, m), x) <= TOL
    assert err(gpu(x[:64], 0), O.sj_apply(x[:64], 0), x[:64]) <= TOL


@pytest.mark.parametrize("shape", [(1024, 1024), (1024, 512), (512, 1024)])
def test_config3_large_arrays(shape):
    h, w = shape
    rng = np.random.default_rng(2)
    yy, xx = np.mgrid[0:h, 0:w]
    x = (rng.standard_normal((h, w)) + np.sin(2 * np.pi * xx / 97) * np.cos(2 * np.pi * yy / 61)).astype(np.float32)
    for m in range(3):
        y = gpu(x[None], m)[0]
        assert err(y, O.fp64_apply(x, m), x) <= TOL
        assert err(y, O.sj_apply(x, m), x) <= TOL


def test_config5_precision_sweep_fp32():
    rng = np.random.default_rng(4)
    mag = 10.0 ** rng.uniform(-6, 6, (2048, 256, 256))
    x = (mag * rng.choice([-1.0, 1.0], size=mag.shape)).astype(np.float32)
    special = rng.choice(2048, 21, replace=False)
    for i, idx in enumerate(special):
        x[idx] = 0
        if i % 2:
            x[idx, rng.integers(256), rng.integers(256)] = 1.0
        else:
            x[idx] = 1.0
    y = gpu(x, 0)
    sub = np.concatenate([special, np.arange(32)])
    assert err(y[sub], O.fp64_apply(x[sub], 0), x[sub]) <= TOL
    rt = gpu(x, 2)
    assert O.rel_max_error(rt, x, x) <= TOL


def test_linearity_and_orthogonality_full_size():
    """Size-independent properties at the largest shape: linearity, Parseval, inverse."""
    rng = np.random.default_rng(11)
    a = rng.standard_normal((4, 1024, 1024)).astype(np.float32)
    b = rng.standard_normal((4, 1024, 1024)).astype(np.float32)
    ya, yb, yab = gpu(a, 0), gpu(b, 0), gpu(a + 2 * b, 0)
    assert np.abs(yab - (ya + 2 * yb)).max() <= 1e-5 * np.abs(yab).max()
    na = np.linalg.norm(a.reshape(4, -1).astype(np.float64), axis=1)
    ny = np.linalg.norm(ya.reshape(4, -1).astype(np.float64), axis=1)
    np.testing.assert_allclose(ny, na, rtol=1e-6)
    back = gpu(ya, 1)
    assert err(back, a, a) <= TOL


def test_blocks8_kernels_agree_bitwise():
    # 8x8 batches run on one of two kernels chosen by batch size and mode (single-buffer tiles of
    # 256 arrays, or double-buffered tiles of 128): the same register program, so the same bits.
    import torch
    from bridct_b200 import torch_api

    big = torch.randn(400000, 8, 8, device="cuda")
    head = big[:3000].clone()
    for mode, n in ((0, 400000), (1, 400000), (2, 200000)):
        y_big = torch_api.apply(big[:n], mode)
        y_small = torch_api.apply(head, mode)
        torch.cuda.synchronize()
        assert torch.equal(y_big[:3000], y_small), mode
        xs = head[:64].cpu().numpy()
        assert O.rel_max_error(y_small[:64].cpu().numpy(), O.fp64_apply(xs, mode), xs, output_scaled=True) <= TOL


@pytest.mark.parametrize("shape,big", [((1024, 1024), 8), ((512, 512), 40), ((1024, 256), 24)])
def test_two_pass_geometries_agree_bitwise(shape, big):
    # A call on few arrays uses narrower column strips and shorter row blocks (more CTAs); the
    # lines themselves are computed the same way, so results match the batch geometry bit for bit.
    x = torch.randn(big, *shape, device="cuda")
    for mode in range(3):
        y_batch = torch_api.apply(x, mode)
        y_one = torch_api.apply(x[:1].clone(), mode)
        torch.cuda.synchronize()
        assert torch.equal(y_batch[:1], y_one), (shape, mode)


@pytest.mark.parametrize("shape", [(8, 16), (8, 32), (8, 64), (16, 8), (16, 16), (16, 32), (16, 64), (32, 16),
                                   (32, 32), (32, 64), (64, 8), (64, 64)])
def test_tile_geometries_agree_bitwise(shape):
    # Batches up to 16 MiB of these shapes run smaller tiles (and 64x64 round trips 128-thread
    # CTAs) than larger batches; every line runs the same register program either way, so a
    # 20 MiB batch and three of its arrays alone agree bit for bit, in every mode.
    h, w = shape
    x = torch.randn((20 << 20) // (4 * h * w), h, w, device="cuda")
    for mode in range(3):
        y_batch = torch_api.apply(x, mode)
        y_few = torch_api.apply(x[:3].clone(), mode)
        torch.cuda.synchronize()
        assert torch.equal(y_batch[:3], y_few), (shape, mode)
    y = torch_api.apply(x[:64], 0).cpu().numpy()
    assert O.rel_max_error(y, O.fp64_apply(x[:64].cpu().numpy(), 0), x[:64].cpu().numpy(), output_scaled=True) <= TOL


@pytest.mark.parametrize("n", [8, 16])
def test_impulse_basis(n):
    # every unit impulse of an n x n array (the reference's impulse-basis tests): each output is
    # a column of the orthonormal 2D transform, so the outputs form an orthogonal matrix
    x = np.zeros((n * n, n, n), np.float32)
    x.reshape(n * n, n * n)[np.arange(n * n), np.arange(n * n)] = 1.0
    for mode in range(3):
        y = torch_api.apply(torch.from_numpy(x).cuda(), mode).cpu().numpy()
        assert O.rel_max_error(y, O.fp64_apply(x, mode), x, output_scaled=True) <= TOL, mode
        m = y.reshape(n * n, n * n).astype(np.float64)
        assert np.abs(m @ m.T - np.eye(n * n)).max() <= 4 * TOL, mode


@pytest.mark.parametrize("shape", [(8, 8), (32, 64), (256, 256), (1024, 128)])
def test_constant_arrays_map_to_dc(shape):
    # a constant array has only a DC coefficient c*sqrt(h*w) (the reference's DC tests)
    h, w = shape
    c = np.float32(-3.75)
    x = np.full((2, h, w), c, np.float32)
    y = torch_api.apply(torch.from_numpy(x).cuda(), 0).cpu().numpy()
    dc = float(c) * np.sqrt(h * w)
    assert np.abs(y[:, 0, 0] - dc).max() <= TOL * abs(dc)
    rest = y.copy()
    rest[:, 0, 0] = 0
    assert np.abs(rest).max() <= TOL * abs(dc)
    back = torch_api.apply(torch.from_numpy(y).cuda(), 1).cpu().numpy()
    assert np.abs(back - c).max() <= TOL * abs(dc)
