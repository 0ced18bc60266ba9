"""Strided batches (bridct_plan_apply_strided_device and the torch entry on views): arrays read and
written where they lie, with row pitches and array strides, for every shape and mode, against
float64 and bitwise against the contiguous path.  The reference accepts contiguous arrays only
(docs/API.md:17); this is the extension that lets sub-images and tensor slices skip a copy."""
import numpy as np
import pytest
import torch

from bridct_b200 import _lib, torch_api
from oracle import oracle as O
from tests.helpers import SHAPES, TOL

pytestmark = pytest.mark.gpu


def _plan(h, w):
    return torch_api._plan(torch.cuda.current_device(), h, w)


def _strided_call(h, w, mode, x, xld, xbs, y, yld, ybs, batch):
    L = _lib.lib()
    return L.bridct_plan_apply_strided_device(_plan(h, w), mode, x.data_ptr(), xld, xbs, y.data_ptr(), yld, ybs,
                                              batch, None)


@pytest.mark.parametrize("h,w", SHAPES)
def test_padded_views_every_shape_and_mode(h, w):
    batch = 3 if h * w <= 65536 else 2
    rng = np.random.default_rng(h * 7 + w)
    big = torch.from_numpy(rng.uniform(-1, 1, (batch, h + 1, w + 12)).astype(np.float32)).cuda()
    xv = big[:, 1:, 4:4 + w]                        # rows w+12 apart, arrays (h+1)(w+12) apart
    xc = xv.contiguous()
    xn = xc.cpu().numpy()
    for mode in range(3):
        obig = torch.full((batch, h + 2, w + 8), float("nan"), device="cuda")
        ov = obig[:, 2:, 4:4 + w]                   # rows w+8 apart, arrays (h+2)(w+8) apart
        st = _strided_call(h, w, mode, xv, w + 12, (h + 1) * (w + 12), ov, w + 8, (h + 2) * (w + 8), batch)
        assert st == 0, _lib.last_error()
        torch.cuda.synchronize()
        got = ov.cpu().numpy()
        exact = O.fp64_apply(xn, mode)
        assert O.rel_max_error(got, exact, xn, output_scaled=True) <= TOL, (h, w, mode)
        ref = torch_api.apply(xc, mode)
        if (h, w) != (8, 8):                        # same kernels, contiguous addressing
            assert torch.equal(ov, ref), (h, w, mode)
        # padding untouched
        assert torch.isnan(obig[:, :2]).all() and torch.isnan(obig[:, 2:, :4]).all()
        assert torch.isnan(obig[:, 2:, 4 + w:]).all()


@pytest.mark.parametrize("h,w", [(8, 8), (32, 64), (256, 128), (1024, 512)])
def test_arrays_side_by_side_in_an_image(h, w):
    """A row of `batch` arrays side by side in one image: array stride w, row pitch batch * w."""
    batch = 4
    img = torch.randn(h, batch * w, device="cuda")
    out = torch.empty_like(img)
    st = _strided_call(h, w, 0, img, batch * w, w, out, batch * w, w, batch)
    assert st == 0, _lib.last_error()
    torch.cuda.synchronize()
    xs = img.view(h, batch, w).permute(1, 0, 2).contiguous().cpu().numpy()
    got = out.view(h, batch, w).permute(1, 0, 2).cpu().numpy()
    assert O.rel_max_error(got, O.fp64_apply(xs, 0), xs, output_scaled=True) <= TOL


def test_strided_rejections_write_nothing():
    h, w, batch = 32, 64, 3
    x = torch.randn(batch * h * (w + 4), device="cuda")
    y = torch.full_like(x, 7.0)
    assert _strided_call(h, w, 0, x, w + 2, h * (w + 2), y, w + 4, h * (w + 4), batch) == _lib.BAD_ALIGNMENT
    assert _strided_call(h, w, 0, x, w - 4, h * w, y, w, h * w, batch) == _lib.INVALID_ARGUMENT
    assert _strided_call(h, w, 0, x, w, 8, y, w, h * w, batch) == _lib.INVALID_ARGUMENT   # arrays overlap
    assert _strided_call(h, w, 0, x, w, h * w, x, w, h * w, batch) == _lib.OVERLAPPING_BUFFERS
    assert _strided_call(h, w, 5, x, w, h * w, y, w, h * w, batch) == _lib.INVALID_ARGUMENT
    torch.cuda.synchronize()
    assert bool((y == 7.0).all())


def test_torch_views_skip_the_copy_and_match():
    base = torch.randn(6, 136, 264, device="cuda")
    v = base[1:5, 4:132, 4:260]                      # 4 arrays of 128 x 256 inside a padded tensor
    assert torch_api._strides(v) == (264, 136 * 264)
    y = torch_api.dct2(v)
    vn = v.contiguous().cpu().numpy()
    assert O.rel_max_error(y.cpu().numpy(), O.fp64_apply(vn, 0), vn, True) <= TOL
    assert torch.equal(y, torch_api.dct2(v.contiguous()))
    # permuted batch axes of a (h, w, b) tensor have no unit column stride -> contiguous copy, same result
    p = torch.randn(64, 64, 4, device="cuda").permute(2, 0, 1)
    assert torch_api._strides(p) is None
    pn = p.contiguous().cpu().numpy()
    assert O.rel_max_error(torch_api.dct2(p).cpu().numpy(), O.fp64_apply(pn, 0), pn, True) <= TOL
    # strided output
    out_base = torch.zeros(4, 130, 260, device="cuda")
    out = out_base[:, 2:, 4:]
    torch_api.apply(v, 1, out=out)
    assert O.rel_max_error(out.cpu().numpy(), O.fp64_apply(vn, 1), vn, True) <= TOL
    assert bool((out_base[:, :2] == 0).all()) and bool((out_base[:, :, :4] == 0).all())
