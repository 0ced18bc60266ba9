"""The NumPy `Plan` contract of the reference (python/test_api.py, python/test_hardening.py,
python/README.md:32-38) on the GPU-backed bridct_b200.bridct_numpy."""
import threading

import numpy as np
import pytest

from bridct_b200 import bridct_numpy
from bridct_b200.bridct_numpy import Plan
from oracle import oracle as O
from tests.helpers import TOL

pytestmark = pytest.mark.gpu

SHAPES = [(8, 8), (16, 32), (8, 64), (64, 64), (128, 16), (256, 256), (1024, 512)]


@pytest.mark.parametrize("shape", SHAPES)
def test_transforms_batches_and_out(shape):
    h, w = shape
    rng = np.random.default_rng(h + w)
    p = Plan(h, w)
    assert p.shape == (h, w) and not p.closed
    assert p.route == ("paper8-square" if h == w and h <= 256 else "blocked-extension")
    for batch in (None, 1, 4):
        x = rng.standard_normal((h, w) if batch is None else (batch, h, w)).astype(np.float32)
        saved = x.copy()
        for name, mode in (("forward", 0), ("inverse", 1), ("roundtrip", 2)):
            y = getattr(p, name)(x)
            assert y.shape == x.shape and y.dtype == np.float32
            assert O.rel_max_error(y, O.fp64_apply(x, mode), x, output_scaled=True) <= TOL
            out = np.empty_like(x)
            r = getattr(p, name)(x, out=out)
            assert r is out and np.array_equal(out, y)
            assert getattr(p, name)(x) is not y
            assert np.array_equal(x, saved)
    p.close()
    assert p.closed and p.route is None


def test_roundtrip_materializes_the_spectrum():
    p = Plan(32, 64)
    x = np.random.default_rng(0).standard_normal((3, 32, 64)).astype(np.float32)
    assert np.array_equal(p.roundtrip(x), p.inverse(p.forward(x)))


@pytest.mark.parametrize("shape", [(3000, 64, 64), (5, 1024, 512), (70000, 8, 8)])
def test_roundtrip_spectrum_on_device_across_pipeline_chunks(shape):
    """Batches of several pipeline chunks: the round trip with the spectrum kept in device staging
    equals a forward call followed by an inverse call, bit for bit."""
    p = Plan(shape[1], shape[2])
    x = np.random.default_rng(1).standard_normal(shape).astype(np.float32)
    assert np.array_equal(p.roundtrip(x), p.inverse(p.forward(x)))


def test_readonly_input_allowed():
    p = Plan(8, 8)
    x = np.ones((8, 8), np.float32)
    x.flags.writeable = False
    p.forward(x)


def test_argument_errors():
    p = Plan(16, 32)
    x = np.zeros((16, 32), np.float32)
    with pytest.raises(TypeError, match="exact NumPy ndarray"):
        p.forward(x.tolist())
    with pytest.raises(TypeError, match="exact NumPy ndarray"):
        p.forward(x.view(np.matrix))
    with pytest.raises(TypeError, match="native-endian float32"):
        p.forward(x.astype(np.float64))
    with pytest.raises(TypeError, match="native-endian float32"):
        p.forward(x.astype(">f4"))
    with pytest.raises(TypeError, match="method\\(input"):
        p.forward(x, np.empty_like(x))
    with pytest.raises(TypeError, match="only accepted keyword"):
        p.forward(x, output=np.empty_like(x))
    with pytest.raises(ValueError, match="batch >= 1"):
        p.forward(np.zeros((32, 16), np.float32))
    with pytest.raises(ValueError, match="batch >= 1"):
        p.forward(np.zeros((0, 16, 32), np.float32))
    with pytest.raises(ValueError, match="batch >= 1"):
        p.forward(np.zeros(512, np.float32))
    with pytest.raises(ValueError, match="C-contiguous"):
        p.forward(np.asfortranarray(x))
    raw = np.zeros(16 * 32 * 4 + 1, np.uint8)
    mis = np.frombuffer(raw.data, dtype=np.float32, count=16 * 32, offset=1).reshape(16, 32)
    with pytest.raises(ValueError, match="C-contiguous, float-aligned"):
        p.forward(mis)
    ro = np.empty_like(x)
    ro.flags.writeable = False
    with pytest.raises(ValueError, match="writable"):
        p.forward(x, out=ro)
    with pytest.raises(ValueError, match="must not overlap"):
        p.forward(x, out=x)
    with pytest.raises(ValueError, match="match exactly"):
        p.forward(np.zeros((2, 16, 32), np.float32), out=np.zeros((3, 16, 32), np.float32))


def test_lifecycle_errors():
    p = Plan(8, 8)
    with pytest.raises(RuntimeError, match="reinitialized"):
        p.__init__(8, 8)
    p._busy = True
    with pytest.raises(RuntimeError, match="another thread"):
        p.forward(np.zeros((8, 8), np.float32))
    with pytest.raises(RuntimeError, match="already initializing or executing"):
        p.close()
    p._busy = False
    p.close()
    p.close()
    with pytest.raises(RuntimeError, match="closed or uninitialized"):
        p.forward(np.zeros((8, 8), np.float32))
    assert bridct_numpy.core_version == "0.2.0-dev.7"


def test_one_plan_per_thread():
    x = np.random.default_rng(1).standard_normal((4, 64, 64)).astype(np.float32)
    want = Plan(64, 64).forward(x)
    bad = []

    def work():
        p = Plan(64, 64)
        for _ in range(20):
            if not np.array_equal(p.forward(x), want):
                bad.append(1)

    ts = [threading.Thread(target=work) for _ in range(4)]
    [t.start() for t in ts]
    [t.join() for t in ts]
    assert not bad
