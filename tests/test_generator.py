"""The SJ generator: float64 exactness of every generated program, and the committed
header is what the generator produces."""
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT / "bridct_b200" / "csrc"))
import gen_sj  # noqa: E402


def test_generated_header_is_current():
    assert (ROOT / "bridct_b200" / "csrc" / "sj_generated.cuh").read_text() == gen_sj.generate() + "\n"


@pytest.mark.parametrize("n", gen_sj.REG_SIZES)
def test_line_programs_exact(n):
    (g, fwd), (gi, inv), (gr, rt) = gen_sj.build_line_ops(n)
    rng = np.random.default_rng(n)
    x = rng.standard_normal((n, 3))
    q = gen_sj._dct_matrix(n)
    assert np.abs(g.evaluate(fwd, x) - q @ x).max() < 1e-11
    assert np.abs(gi.evaluate(inv, np.concatenate([x, np.zeros_like(x)])) - q.T @ x).max() < 1e-11
    assert np.abs(gr.evaluate(rt, x) - x).max() < 1e-11


def test_scaled_core_operation_counts():
    # The scaled SJ 8-point core of the reference (rect_generated.inc:5-104: leaf8 + post8)
    # uses 26 additions and 8 multiplications; the generated one must not be worse.
    g = gen_sj.Graph()
    core = gen_sj.dct2_core(g, [g.inp(i) for i in range(8)])
    c = g.count_ops(core)
    assert c["add"] <= 26 and c["mul"] <= 8


@pytest.mark.parametrize("n", gen_sj.STAGE2_SIZES)
def test_cfft_and_transpose(n):
    (g, outs), (gt, back) = gen_sj.build_cfft(n)
    rng = np.random.default_rng(n)
    z = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    flat = np.stack([z.real, z.imag], 1).reshape(-1, 1)
    got = g.evaluate(outs, flat).reshape(n, 2)
    want = np.fft.fft(z) / np.array([gen_sj.sj_scale(n, k) for k in range(n)])
    assert np.abs(got[:, 0] + 1j * got[:, 1] - want).max() < 1e-11
    yv = rng.standard_normal((2 * n, 1))
    aty = gt.evaluate(back, np.concatenate([yv, np.zeros((2 * n, 1))]))
    assert abs(got.reshape(-1) @ yv[:, 0] - flat[:, 0] @ aty[:, 0]) < 1e-9
