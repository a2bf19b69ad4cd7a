"""Pin the Anderson oracle against the reference's own golden vectors: the
Toth--Kelley residual histories of the aasol docstring
(src/utils/anderson.jl:116-160) and the assertions of test/test_anderson.jl."""
import numpy as np
import pytest

from oracle.anderson import aasol

# anderson.jl:126-135 (beta = 1) and :151-159 (beta = 0.5)
HIST_BETA1 = [6.50111e-01, 4.48661e-01, 2.61480e-02, 7.25389e-02, 1.53107e-04, 1.18513e-05, 1.82466e-08, 1.04725e-13]
COND_BETA1 = [1.00000e00, 2.01556e10, 1.37776e09, 3.61348e10, 2.54948e11, 3.67694e10]
ALPHA_BETA1 = [1.00000e00, 4.61720e00, 2.15749e00, 1.18377e00, 1.00000e00, 1.00171e00]
HIST_BETA05 = [3.25055e-01, 3.70140e-02, 1.81111e-03, 9.55308e-04, 1.25936e-05, 1.40854e-09, 2.18196e-12]


def tothk(u):
    G = np.zeros(2)
    G[0] = np.cos(0.5 * (u[0] + u[1]))
    G[1] = G[0] + 1.0e-8 * np.sin(u[0] * u[0])
    return G


def _check_history(h, golden):
    assert len(h) == len(golden)
    # every entry above the rounding floor of this ill-conditioned problem
    # (condition numbers up to 2.5e11) agrees to 6e-5 relative
    np.testing.assert_allclose(h[:-1], golden[:-1], rtol=6e-5)
    assert h[-1] < 1e-10 and golden[-1] < 1e-10


def test_toth_kelley_beta1():
    out = aasol(tothk, np.ones(2), 2, rtol=1e-10)
    _check_history(out.history, HIST_BETA1)
    np.testing.assert_allclose(out.condhist, COND_BETA1, rtol=1e-3)
    np.testing.assert_allclose(out.alphanorm, ALPHA_BETA1, rtol=1e-5)
    assert out.idid and out.errcode == 0
    np.testing.assert_allclose(out.solution, out.functionval, atol=1e-8)


def test_toth_kelley_beta05():
    out = aasol(tothk, np.ones(2), 2, rtol=1e-10, beta=0.5)
    _check_history(out.history, HIST_BETA05)
    assert out.idid and out.errcode == 0


def test_toth_kelley_picard_warmup():
    # test/test_anderson.jl:30-36
    out = aasol(tothk, np.ones(2), 2, picard_maxit=5, picard_beta=0.5, rtol=1e-10)
    assert out.idid and out.errcode == 0 and out.history[-1] < 1e-10


def test_errcodes():
    # -1: initial iterate already within tolerance
    out = aasol(lambda u: u.copy(), np.ones(3), 2, rtol=1e-10)
    assert out.errcode == -1 and out.idid
    # 10: maxit reached
    out = aasol(tothk, np.ones(2), 2, rtol=1e-30, atol=1e-30, maxit=3)
    assert out.errcode == 10 and not out.idid
    # -2: divergence guard (||r|| >= 1e4 ||r0||)
    out = aasol(lambda u: 10.0 * u + 1.0, np.ones(2), 0, rtol=1e-10, maxit=50)
    assert out.errcode == -2 and not out.idid


@pytest.mark.parametrize("m", [1, 3, 5])
def test_depths_converge_linear_map(m):
    rng = np.random.default_rng(m)
    A = rng.standard_normal((20, 20)) * 0.05
    b = rng.standard_normal(20)
    out = aasol(lambda x: A @ x + b, np.zeros(20), m, rtol=1e-12, atol=1e-12, maxit=100)
    x = np.linalg.solve(np.eye(20) - A, b)
    assert out.idid
    np.testing.assert_allclose(out.solution, x, rtol=1e-9, atol=1e-10)
