"""PyTorch entry point: CUDA tensors, leading batch dimensions, streams and autograd."""
import numpy as np
import pytest
import torch

from bridct_b200 import torch_api
from oracle import oracle as O
from tests.helpers import TOL

pytestmark = pytest.mark.gpu


def test_dct2_idct2_batch_dims():
    x = torch.randn(2, 3, 32, 128, device="cuda")
    y = torch_api.dct2(x)
    xn = x.cpu().numpy().reshape(-1, 32, 128)
    assert O.rel_max_error(y.cpu().numpy().reshape(-1, 32, 128), O.fp64_apply(xn, 0), xn, True) <= TOL
    back = torch_api.idct2(y)
    assert O.rel_max_error(back.cpu().numpy().reshape(-1, 32, 128), xn, xn) <= TOL
    rt = torch_api.roundtrip2(x)
    assert torch.allclose(rt, x, atol=2e-6 * x.abs().max().item())


def test_noncontiguous_and_side_stream():
    x = torch.randn(64, 64, 4, device="cuda").permute(2, 0, 1)
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        y = torch_api.dct2(x)
    s.synchronize()
    xn = x.contiguous().cpu().numpy()
    assert O.rel_max_error(y.cpu().numpy(), O.fp64_apply(xn, 0), xn, True) <= TOL


def test_autograd_is_the_transpose():
    x = torch.randn(3, 16, 64, device="cuda", requires_grad=True)
    w = torch.randn(3, 16, 64, device="cuda")
    (torch_api.dct2(x) * w).sum().backward()
    wn = w.cpu().numpy()
    assert O.rel_max_error(x.grad.cpu().numpy(), O.fp64_apply(wn, 1), wn, True) <= TOL
    x.grad = None
    (torch_api.idct2(x) * w).sum().backward()
    assert O.rel_max_error(x.grad.cpu().numpy(), O.fp64_apply(wn, 0), wn, True) <= TOL


def test_errors():
    with pytest.raises(ValueError):
        torch_api.dct2(torch.zeros(8, 8))
    with pytest.raises(TypeError):
        torch_api.dct2(torch.zeros(8, 8, device="cuda", dtype=torch.float64))
    with pytest.raises(ValueError):
        torch_api.dct2(torch.zeros(8, 12, device="cuda"))
