"""The Newton iteration of the device coexistence solve (saturation_kernel, csrc/bulk.cuh),
restated on the CPU with the host bulk equations, against the oracle's saturation solve
(oracle/pcsaft_bulk.py saturation_pure, Newton with a finite-difference Jacobian).

The device step is, for y = (ln rho_l, ln rho_v), F1 = rho_l Z_l - rho_v Z_v and
F2 = g_l - g_v (g = mu_res / kT + ln rho), with P' = d(p / kT) / d rho from Gibbs-Duhem:
  dy_l = (rho_v F2 - F1) / (P'_l (rho_v - rho_l)),  dy_v = (rho_l F2 - F1) / (P'_v (rho_v - rho_l)),
halved until no component exceeds 0.5, from the densest root at 1e3 Pa and the ideal-gas
vapour there.  No GPU."""
import numpy as np
import pytest

import _systems as S

R = 8.314462618


def newton_like_the_device(pm, T, p_start=1e3):
    def P(r):   # p / RT (mol/m^3)
        return pm.pressure([r], T) / (R * T)

    def g(r):
        return pm.mu_res([r], T)[0] + np.log(r)

    def dP(r):
        h = 1e-5 * r
        return (P(r + h) - P(r - h)) / (2 * h)

    yl = np.log(pm.molar_density(p_start, T, [1.0], "liquid"))
    yv = np.log(p_start / (R * T))
    for it in range(100):
        rl, rv = np.exp(yl), np.exp(yv)
        F1, F2 = P(rl) - P(rv), g(rl) - g(rv)
        dl = (rv * F2 - F1) / (dP(rl) * (rv - rl))
        dv = (rl * F2 - F1) / (dP(rv) * (rv - rl))
        lam = 1.0
        while max(abs(lam * dl), abs(lam * dv)) > 0.5:
            lam *= 0.5
        yl -= lam * dl
        yv -= lam * dv
        if max(abs(dl), abs(dv)) < 1e-13:
            return np.exp(yl), np.exp(yv), it + 1
    raise AssertionError("no convergence")


@pytest.mark.parametrize("name,T", [("octane", 250.0), ("octane", 450.0), ("methane", 150.0), ("water", 373.15)])
def test_gibbs_duhem_newton_reaches_the_oracle_coexistence(name, T):
    from oracle import pcsaft_bulk as pb
    pm, om = S.models([name])
    rl, rv, its = newton_like_the_device(pm, T)
    _, wl, wv = pb.saturation_pure(om, T)
    np.testing.assert_allclose([rl, rv], [wl, wv], rtol=1e-10)
    # the vapour side's pressure, which the device reports, agrees closely; the liquid side's
    # amplifies the last bits of rho_l by 1 / Z_l (about 2e5 for octane at 250 K)
    assert pm.pressure([rv], T) == pytest.approx(pb.pressure(om, [wv], T), rel=1e-10)
    assert its < 30
