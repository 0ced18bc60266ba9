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


@pytest.mark.parametrize("form", ["tc_bf16x3", "tc_tf32x3"])
def test_tensor_core_form_on_two_streams_of_one_cached_plan(form):
    """Two side streams run the same shape's tensor-core form at once through the one cached
    plan: each call's intermediate comes from torch's allocator on its own stream, so the results
    equal the same calls made one at a time."""
    xa = torch.randn(512, 128, 256, device="cuda")
    xb = torch.randn(512, 128, 256, device="cuda")
    ref_a = torch_api.apply(xa, 0, form=form)
    ref_b = torch_api.apply(xb, 0, form=form)
    torch.cuda.synchronize()
    s1, s2 = torch.cuda.Stream(), torch.cuda.Stream()
    outs = []
    for _ in range(3):
        with torch.cuda.stream(s1):
            ya = torch_api.apply(xa, 0, form=form)
        with torch.cuda.stream(s2):
            yb = torch_api.apply(xb, 0, form=form)
        outs.append((ya, yb))
    torch.cuda.synchronize()
    for ya, yb in outs:
        assert torch.equal(ya, ref_a) and torch.equal(yb, ref_b)


def test_calls_leave_the_current_device_unchanged():
    dev = torch.cuda.current_device()
    x = torch.randn(4, 256, 256, device=f"cuda:{dev}")
    torch_api.dct2(x)
    torch_api.apply(x, 0, form="tc_bf16x3")
    torch.cuda.synchronize()
    assert torch.cuda.current_device() == dev


def test_apply_sharded_over_the_visible_devices():
    """One process splitting a batch over every visible GPU (each shard on its own device) gives
    the single-call result."""
    from bridct_b200.dist import apply_sharded

    x = torch.randn(13, 64, 128, device="cuda")
    devs = list(range(torch.cuda.device_count())) * 2       # with one GPU: two shards on it
    y = apply_sharded(x, 0, devices=devs)
    assert torch.equal(y, torch_api.apply(x, 0))
    xn = x.cpu().numpy()
    yn = apply_sharded(xn, 1, devices=devs)
    assert isinstance(yn, np.ndarray)
    assert O.rel_max_error(yn, O.fp64_apply(xn, 1), xn, True) <= TOL
