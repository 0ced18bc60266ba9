"""The ragged-batch entry point that allocates nothing (bridct_ragged_apply_noalloc).

It exists for callers that cannot let a library allocate device memory: a framework whose
caching allocator owns the whole GPU, a loop that cannot afford cudaMalloc's implicit device
synchronisation, or a process with a fixed device footprint.  The entry point keeps its work
queue, counters and tables in one static device array.  These tests call it through the C-ABI
twice in a row, with different batches, and compare each result with the allocating entry
point (bridct_ragged_create + bridct_ragged_apply_device) within the parity bound, and a sample
of each call's arrays (the 1024x1024 two-pass array, four-step arrays with 128/256/512 axes and
small tiles) directly with the float64 transform.  The file is collected last, and passes both
alone in a fresh process and after the other tests.
"""
import numpy as np
import pytest
import torch

from bridct_b200 import _lib
from bridct_b200.ragged import RaggedBatch
from oracle import oracle as O
from tests.helpers import SIZES, TOL

pytestmark = pytest.mark.gpu


def _items(seed, n):
    rng = np.random.default_rng(seed)
    out = [(int(rng.choice(SIZES)), int(rng.choice(SIZES)), int(rng.integers(0, 3))) for _ in range(n)]
    out += [(1024, 1024, 0), (8, 8, 1), (128, 1024, 2)]       # two-pass, tile and rect arrays
    out += [(128, 256, 1), (256, 512, 0), (512, 128, 2)]      # four-step lines of every width
    return out


def _fp64_sample(items):
    """Indices checked against float64: the appended arrays plus every 15th random one."""
    return sorted(set(range(len(items) - 6, len(items))) | set(range(0, len(items) - 6, 15)))


def _c_items(batch):
    arr = (_lib.RaggedItem * len(batch.items))()
    for i, ((h, w, m), o) in enumerate(zip(batch.items, batch.offsets)):
        arr[i] = _lib.RaggedItem(h, w, m, 0, int(o))
    return arr


def test_noalloc_matches_allocating_entry_point_on_two_calls():
    L = _lib.lib()
    for seed in (21, 22):                      # two calls in a row, different batches
        items = _items(seed, 90)
        ref_batch = RaggedBatch(items)
        x = torch.from_numpy(np.random.default_rng(seed).uniform(-1, 1, ref_batch.span).astype(np.float32)).cuda()
        ref = ref_batch.apply(x)
        y = torch.full_like(x, float("nan"))
        torch.cuda.synchronize()
        st = L.bridct_ragged_apply_noalloc(_c_items(ref_batch), len(items), x.data_ptr(), y.data_ptr(), None)
        assert st == _lib.OK, _lib.last_error()
        for (h, w, m), xi, yi, ri in zip(items, ref_batch.unpack(x), ref_batch.unpack(y), ref_batch.unpack(ref)):
            xi, yi, ri = xi.cpu().numpy(), yi.cpu().numpy(), ri.cpu().numpy()
            assert np.isfinite(yi).all(), (h, w, m)
            assert O.rel_max_error(yi, ri, xi, output_scaled=True) <= TOL, (h, w, m)
        xs, ys = ref_batch.unpack(x), ref_batch.unpack(y)
        for i in _fp64_sample(items):
            h, w, m = items[i]
            xi, yi = xs[i].cpu().numpy(), ys[i].cpu().numpy()
            assert O.rel_max_error(yi, O.fp64_apply(xi, m), xi, output_scaled=True) <= TOL, (h, w, m)


def test_noalloc_rejects_batches_beyond_its_maximum():
    L = _lib.lib()
    n = 4097
    arr = (_lib.RaggedItem * n)()
    for i in range(n):
        arr[i] = _lib.RaggedItem(8, 8, 0, 0, 64 * i)
    x = torch.zeros(64 * n, device="cuda")
    y = torch.zeros_like(x)
    assert L.bridct_ragged_apply_noalloc(arr, n, x.data_ptr(), y.data_ptr(), None) == _lib.INVALID_ARGUMENT
    assert "4096" in _lib.last_error()
    assert bool((y == 0).all())
