"""The DDFT right-hand side (ext/SciMLBasecDFTExt.jl:10-61) on the CPU.

The device applies the spectral maps of ddft_rhs_log! as periodic circulants along each
axis, with taps from the exact-reduction formula of ddft_axis_taps (csrc/cdft_b200.cu).
This file emulates that operator in NumPy and checks it against the oracle's FFT form
(convolve!, integrals.jl:88-96) on random fields, odd and even lengths, 1D and 3D."""
import numpy as np
import pytest

from oracle import functional as fn


def _axis_taps(n, B):
    """NumPy copy of ddft_axis_taps: real inverse DFT of 2 pi i m/B and -(2 pi m/B)^2."""
    m = np.fft.fftfreq(n) * n
    q = np.arange(n)
    r = np.mod(np.outer(q, m).astype(np.int64), n)
    th = 2 * np.pi * r / n
    sn, cs = np.sin(th), np.cos(th)
    sn[(r == 0) | (2 * r == n)] = 0.0
    cs[(4 * r == n) | (4 * r == 3 * n)] = 0.0
    tg = -(2 * np.pi / (n * B)) * (sn * m).sum(axis=1)
    tl = -((2 * np.pi) ** 2 / (n * B * B)) * (cs * m * m).sum(axis=1)
    return tg, tl


def _circ(x, t, axis):
    """out[j] = sum_q t[q] x[(j - q) mod n] along ``axis``."""
    n = x.shape[axis]
    out = np.zeros_like(x)
    for q in range(n):
        out += t[q] * np.roll(x, q, axis=axis)
    return out


def _emulated_rhs(eta, mu, boxes):
    nd = len(boxes)
    out = np.zeros_like(eta)
    for d in range(nd):
        axis = eta.ndim - 1 - d          # x is the last axis
        tg, tl = _axis_taps(eta.shape[axis], boxes[d])
        ge, gm = _circ(eta, tg, axis), _circ(mu, tg, axis)
        out += _circ(eta + mu, tl, axis) + ge * ge + gm * ge
    return out


class _Fake:
    """The parts of the oracle's DFTSystem that ddft_rhs uses, with mu given."""

    def __init__(self, shape, boxes, L, mu):
        nd = len(boxes)
        self.nc = shape[0]
        self.nd = nd
        self.L = L
        self._mu = mu
        self.structure = fn.Structure((1e5, 300.0), [1.0] * self.nc, [(0.0, b * L) for b in boxes],
                                      tuple(reversed(shape[1:])))

    _omega = fn.DFTSystem._omega
    _conv = fn.DFTSystem._conv
    ddft_rhs = fn.DFTSystem.ddft_rhs

    def dFdrho(self, rho):
        return self._mu


@pytest.mark.parametrize("shape,boxes", [((2, 64), (7.3,)), ((1, 63), (5.1,)), ((1, 8, 6, 10), (4.0, 3.3, 5.5)),
                                         ((1, 7, 7, 7), (3.0, 3.0, 3.0))])
def test_axis_circulants_equal_the_fft_maps(shape, boxes):
    rng = np.random.default_rng(4)
    eta = rng.standard_normal(shape)
    mu = rng.standard_normal(shape)
    fake = _Fake(shape, boxes, 3.4e-10, mu)
    want = fake.ddft_rhs(eta)
    got = _emulated_rhs(eta, mu, boxes)
    np.testing.assert_allclose(got, want, rtol=0, atol=1e-11 * np.max(np.abs(want)))
