"""The CPU oracle (oracle/sj_oracle.c) pinned against the reference's own outputs.

The golden fixtures hold the reference library's outputs (tests/golden/make_golden.py); the
float64 Q-matrix contract is the second, independent pin.
"""
import numpy as np
import pytest

from oracle import oracle as O
from tests.helpers import FROB, SIZES, TOL, corpus_files, frob_rel, golden, verify_files

# plan_scale(8, k) = sj_scale(32, k) sqrt((k ? 2 : 1)/8): the reference's scale8 table
# (src/generated/rect_generated.inc:115), a known answer for the scale recursion.
SCALE8 = [0.35355339059327379, 0.34675996133053688, 0.46193976625564337, 0.29396890060483971,
          0.35355339059327379, 0.29396890060483971, 0.46193976625564337, 0.34675996133053688]


def test_sj_scale_known_answer():
    got = [O.sj_scale(32, k) * np.sqrt((2.0 if k else 1.0) / 8) for k in range(8)]
    np.testing.assert_allclose(got, SCALE8, rtol=1e-15)
    assert O.sj_scale(4, 3) == 1.0 and O.sj_scale(8, 1) == pytest.approx(np.cos(np.pi / 4))


@pytest.mark.parametrize("n", SIZES)
def test_core_is_scaled_dct2_and_transpose(n):
    rng = np.random.default_rng(n)
    q = O.q_matrix(n)
    s = np.array([O.sj_scale(4 * n, k) * np.sqrt((2.0 if k else 1.0) / n) for k in range(n)])
    x = rng.standard_normal(n).astype(np.float32)
    want = (q @ x.astype(np.float64)) / s
    assert np.abs(O.sj_core(x) - want).max() <= 4e-7 * np.abs(want).max()
    want_t = (q / s[:, None]).T @ x.astype(np.float64)
    assert np.abs(O.sj_core(x, transpose=True) - want_t).max() <= 4e-7 * np.abs(want_t).max()


@pytest.mark.parametrize("path", corpus_files(), ids=lambda p: p.stem)
def test_oracle_matches_reference_corpus(path):
    g = golden(path.name)
    x, dom = g["x"], g["domain"]
    core = dom == "core"
    for m in range(3):
        y = O.sj_apply(x, m)
        ref = g[f"y{m}"]
        exact = O.fp64_apply(x, m)
        # max-norm error scaled by max(|x|, |ref|): DC-heavy corpus cases have outputs n times
        # larger than the input, where the reference itself is ~1e-5 off in max|err|/max|x|.
        assert O.rel_max_error(y[core], ref[core], x[core], output_scaled=True) <= TOL
        assert O.rel_max_error(y[core], exact[core], x[core], output_scaled=True) <= TOL
        assert O.rel_max_error(ref[core], exact[core], x[core], output_scaled=True) <= TOL
        for i in np.where(core)[0]:
            assert frob_rel(y[i], exact[i], x[i]) < FROB


@pytest.mark.parametrize("path", verify_files(), ids=lambda p: p.stem)
def test_oracle_matches_reference_verify_families(path):
    g = golden(path.name)
    x = g["x"]
    for m in range(3):
        y = O.sj_apply(x, m)
        assert np.isfinite(y).all()
        assert O.rel_max_error(y, g[f"y{m}"], x, output_scaled=True) <= TOL
        assert O.rel_max_error(y, O.fp64_apply(x, m), x, output_scaled=True) <= TOL


def test_oracle_matches_reference_configs():
    g = golden("configs.npz")
    for key in ("c1", "c2", "c3", "c5"):
        x = g[f"{key}_x"]
        for m in range(3):
            y = O.sj_apply(x, m)
            assert O.rel_max_error(y, g[f"{key}_y{m}"], x, output_scaled=True) <= TOL


@pytest.mark.skipif(not O.ref_available(), reason="reference library not built here")
@pytest.mark.parametrize("h", SIZES)
def test_oracle_matches_live_reference_all_shapes(h):
    rng = np.random.default_rng(h)
    for w in SIZES:
        x = rng.uniform(-1, 1, (1, h, w)).astype(np.float32)
        for m in range(3):
            assert O.rel_max_error(O.sj_apply(x, m), O.ref_apply(x, m), x, output_scaled=True) <= TOL


def test_oracle_rejects_unsupported():
    with pytest.raises(ValueError):
        O.sj_apply(np.zeros((32, 26), np.float32), 0)
