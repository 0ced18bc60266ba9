"""Batching form: one persistent launch over mixed shapes and directions, against float64 per
array, the per-array launch loop and other unit geometries (all within the parity bound)."""
import numpy as np
import pytest
import torch

from bridct_b200.ragged import RaggedBatch
from oracle import oracle as O
from tests.helpers import SIZES, TOL

pytestmark = pytest.mark.gpu


def random_batch(n, seed, max_elems=1 << 20):
    rng = np.random.default_rng(seed)
    items = []
    while len(items) < n:
        h, w = int(rng.choice(SIZES)), int(rng.choice(SIZES))
        if h * w <= max_elems:
            items.append((h, w, int(rng.integers(0, 3))))
    return items


@pytest.mark.parametrize("seed", [0, 1])
def test_ragged_all_shapes_vs_fp64(seed):
    items = random_batch(160, seed)
    items += [(h, w, m) for h in SIZES for w in SIZES for m in (0, 1) if (h * w) <= 65536][: 40]
    b = RaggedBatch(items)
    rng = np.random.default_rng(seed + 10)
    x = torch.from_numpy(rng.uniform(-1, 1, b.span).astype(np.float32)).cuda()
    y = b.apply(x)
    torch.cuda.synchronize()
    assert not b.timed_out()
    ys = [t.cpu().numpy() for t in b.unpack(y)]
    xs = [t.cpu().numpy() for t in b.unpack(x)]
    for (h, w, m), xi, yi in zip(items, xs, ys):
        assert O.rel_max_error(yi, O.fp64_apply(xi, m), xi, output_scaled=True) <= TOL, (h, w, m)


def close(a, b, x, items, batch):
    for (h, w, m), xa, ya, yb in zip(items, batch.unpack(x), batch.unpack(a), batch.unpack(b)):
        xa, ya, yb = xa.cpu().numpy(), ya.cpu().numpy(), yb.cpu().numpy()
        assert O.rel_max_error(ya, yb, xa, output_scaled=True) <= TOL, (h, w, m)


def test_ragged_matches_launch_loop():
    items = random_batch(120, 5)
    b = RaggedBatch(items)
    x = torch.randn(b.span, device="cuda")
    y1 = b.apply(x)
    y2 = b.apply_loop(x)
    torch.cuda.synchronize()
    assert not b.timed_out()
    close(y1, y2, x, items, b)


@pytest.mark.parametrize("tuning", [dict(tile_floats=4096, strip_floats=4096, row_floats=4096, lookahead=1),
                                    dict(tile_floats=16384, strip_floats=8192, row_floats=16384, lookahead=8),
                                    dict(tile_floats=1024, strip_floats=2048, row_floats=2048, lookahead=16)])
def test_ragged_tunings_agree(tuning):
    items = random_batch(60, 9)
    x = torch.randn(RaggedBatch(items).span, device="cuda")
    b = RaggedBatch(items)
    ref = b.apply(x)
    got = RaggedBatch(items, tuning=tuning).apply(x)
    torch.cuda.synchronize()
    close(ref, got, x, items, b)


def test_ragged_graph_capture_and_replay():
    items = random_batch(64, 3)
    b = RaggedBatch(items)
    x = torch.randn(b.span, device="cuda")
    y = torch.empty_like(x)
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        b.apply(x, y)
    s.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=s):
        b.apply(x, y, stream=s.cuda_stream)
    y.zero_()
    with torch.cuda.stream(s):
        g.replay()
        g.replay()
    s.synchronize()
    ref = b.apply(x)
    torch.cuda.synchronize()
    assert torch.equal(y, ref)          # the same kernel, replayed from the graph


def test_ragged_rejects_bad_items():
    with pytest.raises(ValueError):
        RaggedBatch([(8, 12, 0)])
    with pytest.raises(ValueError):
        RaggedBatch([(8, 8, 0), (8, 8, 0)], offsets=[0, 32])     # overlap
    with pytest.raises(ValueError):
        RaggedBatch([(8, 8, 0)], offsets=[2])                    # misaligned


def test_autotune_picks_a_measured_geometry():
    from bridct_b200.autotune import tune

    items = random_batch(48, 5)
    x = torch.randn(RaggedBatch(items).span, device="cuda")
    cands = {"tile_floats": (4096, 16384), "lookahead": (1, 4)}
    res = tune(items, x, candidates=cands, sweeps=1, steps=2)
    assert res["best_ms"] <= res["default_ms"]
    assert len(res["table"]) >= 3
    assert all(k in res["best"] for k in ("tile_floats", "strip_floats", "row_floats", "lookahead"))
    b = RaggedBatch(items)
    ref = b.apply(x)
    got = RaggedBatch(items, tuning=res["best"]).apply(x)
    torch.cuda.synchronize()
    close(ref, got, x, items, b)


def test_ragged_dependency_wait_expires_and_reports():
    """The row blocks' bounded wait on their column strips: with a wait limit of zero polls every
    row block gives up at once, skips its rows and raises the batch's flag; the kernel still
    returns, the flag reads nonzero once and then clears, tile arrays are unaffected, and with
    the default limit restored the same batch transforms correctly."""
    from bridct_b200 import _lib

    L = _lib.lib()
    items = [(8, 8, 0), (64, 64, 1), (256, 512, 0), (1024, 128, 1), (32, 16, 2), (512, 512, 0)]
    b = RaggedBatch(items)
    rng = np.random.default_rng(7)
    x = torch.from_numpy(rng.uniform(-1, 1, b.span).astype(np.float32)).cuda()
    y = torch.zeros_like(x)
    assert L.bridct_ragged_set_wait_limit(b._h, 0) == 0
    b.apply(x, y)
    torch.cuda.synchronize()                  # the kernel returned
    assert b.timed_out()
    assert not b.timed_out()                  # read and cleared
    for (h, w, m), xi, yi in zip(items, b.unpack(x), b.unpack(y)):
        if h * w <= 16384:                    # whole-array units never wait
            xi, yi = xi.cpu().numpy(), yi.cpu().numpy()
            assert O.rel_max_error(yi, O.fp64_apply(xi, m), xi, output_scaled=True) <= TOL, (h, w, m)
    assert L.bridct_ragged_set_wait_limit(b._h, 1 << 22) == 0
    y = b.apply(x)
    torch.cuda.synchronize()
    assert not b.timed_out()
    for (h, w, m), xi, yi in zip(items, b.unpack(x), b.unpack(y)):
        xi, yi = xi.cpu().numpy(), yi.cpu().numpy()
        assert O.rel_max_error(yi, O.fp64_apply(xi, m), xi, output_scaled=True) <= TOL, (h, w, m)


def _all(b, kind):
    return {c["key"]: kind for c in b.classes()}


@pytest.mark.parametrize("kind,streams", [("launch", 1), ("launch", 4), ("launch_small", 8), ("mixed", 3)])
def test_class_schedules_match_the_queue_and_fp64(kind, streams):
    items = random_batch(200, 11)
    items += [(1024, 1024, 0), (1024, 1024, 1), (512, 256, 2), (8, 8, 0), (8, 8, 1)]
    b = RaggedBatch(items)
    rng = np.random.default_rng(12)
    x = torch.from_numpy(rng.uniform(-1, 1, b.span).astype(np.float32)).cuda()
    ref = b.apply(x)
    torch.cuda.synchronize()
    classes = b.classes()
    assert sum(c["arrays"] for c in classes) == len(items)
    assert [c["h"] * c["w"] * c["arrays"] for c in classes] == sorted(
        (c["h"] * c["w"] * c["arrays"] for c in classes), reverse=True)
    if kind == "mixed":
        sched = {c["key"]: ("queue", "launch", "launch_small")[i % 3] for i, c in enumerate(classes)}
    else:
        sched = _all(b, kind)
    s = RaggedBatch(items, schedule={"classes": sched, "streams": streams})
    assert all(c["schedule"] == {"queue": 0, "launch": 1, "launch_small": 2}[sched[c["key"]]] for c in s.classes())
    y = s.apply(x)
    torch.cuda.synchronize()
    assert not s.timed_out()
    close(y, ref, x, items, b)
    for i in range(0, len(items), 17):
        h, w, m = items[i]
        xi, yi = b.unpack(x)[i].cpu().numpy(), b.unpack(y)[i].cpu().numpy()
        assert O.rel_max_error(yi, O.fp64_apply(xi, m), xi, output_scaled=True) <= TOL, (h, w, m)


def test_class_schedule_graph_capture_and_replay():
    items = random_batch(96, 13)
    b = RaggedBatch(items)
    b.set_schedule({"classes": {c["key"]: ("launch" if i % 2 else "queue") for i, c in enumerate(b.classes())},
                    "streams": 4})
    x = torch.randn(b.span, device="cuda")
    y = torch.empty_like(x)
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        b.apply(x, y, stream=s.cuda_stream)
    s.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=s):
        b.apply(x, y, stream=s.cuda_stream)
    y.zero_()
    with torch.cuda.stream(s):
        g.replay()
    s.synchronize()
    ref = RaggedBatch(items).apply(x)
    torch.cuda.synchronize()
    close(y, ref, x, items, b)


def test_class_schedule_rejects_bad_arguments():
    from bridct_b200 import _lib
    import ctypes as C

    b = RaggedBatch(random_batch(20, 2))
    n = len(b.classes())
    arr = (C.c_int * n)(*([1] * n))
    L = _lib.lib()
    assert L.bridct_ragged_set_schedule(b._h, arr, n + 1, 4) == _lib.INVALID_ARGUMENT
    assert L.bridct_ragged_set_schedule(b._h, arr, n, 9) == _lib.INVALID_ARGUMENT
    bad = (C.c_int * n)(*([3] * n))
    assert L.bridct_ragged_set_schedule(b._h, bad, n, 4) == _lib.INVALID_ARGUMENT
    x = torch.zeros(b.span, device="cuda")
    assert L.bridct_ragged_apply_class_device(b._h, 0, 0, x.data_ptr(), x.data_ptr(), None) == _lib.INVALID_ARGUMENT
    assert L.bridct_ragged_apply_class_device(b._h, n, 1, x.data_ptr(), x.data_ptr(), None) == _lib.INVALID_ARGUMENT


def test_tune_classes_returns_a_checked_schedule():
    from bridct_b200.autotune import tune_classes

    items = random_batch(40, 17, max_elems=1 << 18)
    x = torch.randn(RaggedBatch(items).span, device="cuda")
    res = tune_classes(items, x, steps=2, streams=(1, 4))
    assert res["ms"] <= res["queue_ms"]
    assert len(res["classes"]) == len(RaggedBatch(items).classes())
    b = RaggedBatch(items, schedule=res["schedule"])
    got = b.apply(x)
    ref = RaggedBatch(items).apply(x)
    torch.cuda.synchronize()
    close(got, ref, x, items, b)


@pytest.mark.parametrize("streams", [1, 3, 8])
def test_merged_schedule_matches_queue_and_fp64(streams):
    """Two-pass classes in merged column and row passes (one launch per column length and mode,
    then one per row length and mode), the others in the queue or their own launch."""
    from bridct_b200.ragged import two_pass

    items = random_batch(240, 21)
    items += [(1024, 1024, 0), (1024, 512, 1), (512, 1024, 2), (256, 128, 0), (32, 1024, 2), (1024, 32, 1)]
    b = RaggedBatch(items)
    rng = np.random.default_rng(22)
    x = torch.from_numpy(rng.uniform(-1, 1, b.span).astype(np.float32)).cuda()
    ref = b.apply(x)
    sched = {}
    for i, c in enumerate(b.classes()):
        sched[c["key"]] = "merged" if two_pass(c["h"], c["w"], c["mode"]) else ("launch" if i % 2 else "queue")
    assert "merged" in sched.values()
    m = RaggedBatch(items, schedule={"classes": sched, "streams": streams})
    y = m.apply(x)
    torch.cuda.synchronize()
    assert not m.timed_out()
    close(y, ref, x, items, b)
    for i in range(0, len(items), 11):
        h, w, mo = items[i]
        xi, yi = b.unpack(x)[i].cpu().numpy(), b.unpack(y)[i].cpu().numpy()
        assert O.rel_max_error(yi, O.fp64_apply(xi, mo), xi, output_scaled=True) <= TOL, (h, w, mo)
    # captured and replayed
    s = torch.cuda.Stream()
    y2 = torch.full_like(x, float("nan"))
    with torch.cuda.stream(s):
        m.apply(x, y2, stream=s.cuda_stream)
    s.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=s):
        m.apply(x, y2, stream=s.cuda_stream)
    y2.fill_(float("nan"))
    with torch.cuda.stream(s):
        g.replay()
    s.synchronize()
    assert torch.equal(y2, y)


def test_merged_schedule_rejects_single_pass_classes():
    from bridct_b200 import _lib
    import ctypes as C

    b = RaggedBatch([(64, 64, 0), (1024, 1024, 0)])
    cls = b.classes()
    arr = (C.c_int * len(cls))(*[3 if c["h"] * c["w"] <= 16384 else 0 for c in cls])
    assert _lib.lib().bridct_ragged_set_schedule(b._h, arr, len(cls), 2) == _lib.INVALID_ARGUMENT
    assert "two-pass" in _lib.last_error()


def test_launch_count_matches_the_kernels_one_apply_runs():
    """bridct_ragged_launch_count (the figure bench.py reports as gpu_launches) against the
    kernels the CUDA profiler records for one apply: the queue alone, then a mixed schedule."""
    from torch.profiler import ProfilerActivity, profile

    from bridct_b200.ragged import two_pass

    items = random_batch(120, 31) + [(1024, 1024, 0), (512, 256, 1), (64, 64, 0), (1024, 32, 1)]
    b = RaggedBatch(items)
    x = torch.from_numpy(np.random.default_rng(32).uniform(-1, 1, b.span).astype(np.float32)).cuda()
    sched = {}
    for i, c in enumerate(b.classes()):
        if two_pass(c["h"], c["w"], c["mode"]) and i % 2:
            sched[c["key"]] = "merged"
        else:
            sched[c["key"]] = ("launch", "queue", "launch_small" if c["h"] * c["w"] > 16384 else "launch")[i % 3]
    m = RaggedBatch(items, schedule={"classes": sched, "streams": 4})
    assert b.launch_count() == 1
    for batch in (b, m):
        y = batch.apply(x)
        torch.cuda.synchronize()
        with profile(activities=[ProfilerActivity.CUDA]) as prof:
            batch.apply(x, y)
            torch.cuda.synchronize()
        kernels = [e for e in prof.events() if e.device_type == torch.autograd.DeviceType.CUDA
                   and "memset" not in e.name.lower() and "memcpy" not in e.name.lower()]
        assert len(kernels) == batch.launch_count(), sorted(e.name for e in kernels)
    assert m.launch_count() > 1


def test_apply_ragged_sharded_matches_one_batch():
    """The element split over the GPUs of one process (here device 0 twice) gives the single
    batch's results bit for bit: each array is transformed by the same kernels either way."""
    from bridct_b200.dist import apply_ragged_sharded

    items = random_batch(90, 41)
    b = RaggedBatch(items)
    x = torch.from_numpy(np.random.default_rng(42).uniform(-1, 1, b.span).astype(np.float32)).cuda()
    y_one = b.apply(x)
    y_split = apply_ragged_sharded(items, x, devices=[0, 0])
    torch.cuda.synchronize()
    assert y_split.device == x.device and y_split.shape == x.shape
    assert torch.equal(y_split, y_one)
