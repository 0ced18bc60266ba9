"""In-image 8x8 block transform (strided, in place, optional fused quantization) against
float64 per block, and against the contiguous batch path."""
import numpy as np
import pytest
import torch

from bridct_b200 import _lib, torch_api
from oracle import oracle as O
from tests.helpers import TOL

pytestmark = pytest.mark.gpu

# a step table growing with frequency, as codec tables do (values 3 .. 59)
STEPS = np.fromfunction(lambda u, v: 3.0 + 4.0 * (u + v), (8, 8)).astype(np.float32)


def to_blocks(img):
    h, w = img.shape
    return img.reshape(h // 8, 8, w // 8, 8).transpose(0, 2, 1, 3).reshape(-1, 8, 8)


def from_blocks(b, h, w):
    return b.reshape(h // 8, w // 8, 8, 8).transpose(0, 2, 1, 3).reshape(h, w)


def image(h, w, seed):
    return (np.random.default_rng(seed).integers(0, 256, (h, w)) - 128).astype(np.float32)


@pytest.mark.parametrize("shape", [(8, 8), (64, 1024), (520, 136), (1024, 1024)])
def test_image_blocks_match_fp64(shape):
    h, w = shape
    x = image(h, w, h + w)
    for mode in range(3):
        y = torch_api.image_blocks8(torch.from_numpy(x).cuda(), mode).cpu().numpy()
        ref = from_blocks(O.fp64_apply(to_blocks(x).astype(np.float64), mode), h, w)
        assert O.rel_max_error(y, ref, x) <= TOL, mode


def test_image_blocks_match_contiguous_batch_bitwise():
    # the same register program as the contiguous 8x8 kernel: results agree bit for bit
    x = image(256, 512, 3)
    y = torch_api.image_blocks8(torch.from_numpy(x).cuda(), 0).cpu().numpy()
    yb = torch_api.apply(torch.from_numpy(to_blocks(x).copy()).cuda(), 0).cpu().numpy()
    assert np.array_equal(to_blocks(y), yb)


def test_strided_view_and_in_place():
    big = torch.from_numpy(image(96, 200, 5)).cuda()
    view = big[8:72, 12:140]                       # 64 x 128 sub-image, row pitch 200 floats
    ref = torch_api.image_blocks8(view.contiguous(), 0)
    got = torch_api.image_blocks8(view, 0)
    torch.cuda.synchronize()
    assert torch.equal(got, ref)
    before = big.clone()
    torch_api.image_blocks8(view, 0, out=view)   # in place inside the larger image
    torch.cuda.synchronize()
    assert torch.equal(big[8:72, 12:140], ref)
    outside = torch.ones_like(big, dtype=torch.bool)
    outside[8:72, 12:140] = False
    assert torch.equal(big[outside], before[outside])


def test_quantize_dequantize():
    h, w = 128, 256
    x = image(h, w, 9)
    xb = to_blocks(x).astype(np.float64)
    yq = torch_api.image_blocks8(torch.from_numpy(x).cuda(), 0, quant=STEPS).cpu().numpy()
    exact = O.fp64_apply(xb, 0) / STEPS
    ref = np.rint(exact)
    got = to_blocks(yq)
    # rounding may differ only where the exact quotient lies within float32 error of a half step
    diff = got != ref
    near_half = np.abs(np.abs(exact - np.floor(exact)) - 0.5) < 1e-4
    assert np.all(~diff | near_half) and np.abs(got - ref).max() <= 1
    # dequantize + inverse
    xr = torch_api.image_blocks8(torch.from_numpy(yq).cuda(), 1, quant=STEPS).cpu().numpy()
    ref_r = from_blocks(O.fp64_apply(to_blocks(yq).astype(np.float64) * STEPS, 1), h, w)
    assert O.rel_max_error(xr, ref_r, x, output_scaled=True) <= TOL
    # the fused round trip equals the two calls
    rt = torch_api.image_blocks8(torch.from_numpy(x).cuda(), 2, quant=STEPS).cpu().numpy()
    assert np.abs(rt - xr).max() <= 1e-3 * np.abs(xr).max()


def test_image_rejects_bad_geometry():
    L = _lib.lib()
    t = torch.zeros(16, 16, device="cuda")
    assert L.bridct_image_blocks8_device(0, t.data_ptr(), 16, t.data_ptr(), 16, 12, 16, None, None) == _lib.INVALID_ARGUMENT
    assert L.bridct_image_blocks8_device(0, t.data_ptr(), 14, t.data_ptr(), 16, 8, 8, None, None) == _lib.BAD_ALIGNMENT
    assert L.bridct_image_blocks8_device(0, t.data_ptr(), 16, t.data_ptr() + 64, 16, 8, 8, None, None) == \
        _lib.OVERLAPPING_BUFFERS
    bad_q = np.zeros(64, np.float32)
    assert L.bridct_image_blocks8_device(0, t.data_ptr(), 16, t.data_ptr(), 16, 16, 16, bad_q.ctypes.data,
                                         None) == _lib.INVALID_ARGUMENT
