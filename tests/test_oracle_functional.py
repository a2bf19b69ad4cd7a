"""Pin the functional oracle: bulk consistency against the independent bulk
PC-SAFT (the property test/test_models.jl:11-27,153-188 and
test/test_coordinate_systems.jl:1-33 assert with Clapeyron), kernel moment
identities, and its complex-step derivatives against finite differences."""
import numpy as np
import pytest

from _systems import PARAMS, models
from oracle import functional as fn
from oracle import pcsaft_bulk as pb


def _uniform(names, rho, T, N=3, nd=1, box=10.0):
    _, om = models(names)
    L = om.length_scale()
    st = fn.Structure((1e5, T), rho, [(-box * L, box * L)] * nd, (N,) * nd)
    return om, fn.DFTSystem(om, st)


@pytest.mark.parametrize("names,state", [
    (["methane"], ("liquid", 1e7, 150.0, [1.0])),
    (["water"], ("liquid", 1e5, 298.15, [1.0])),
    (["octane"], ("liquid", 1e5, 298.15, [1.0])),
    (["water", "octane"], ("liquid", 1e5, 298.15, [0.5, 0.5])),
    (["methane", "octane"], ("liquid", 1e6, 250.0, [0.3, 0.7])),
    (["water", "ethanol"], ("liquid", 1e5, 298.15, [0.5, 0.5])),
])
def test_bulk_consistency(names, state):
    """test/test_models.jl:11-27,153-188: delta F/delta rho_res at a uniform profile equals
    the bulk mu_res; water + ethanol takes the general association path with 4 pairs
    (self and cross, assoc.jl:771-828) as the reference's water+ethanol case does."""
    phase, p, T, x = state
    _, om = models(names)
    x = np.asarray(x)
    rho = x * pb.density(om, p, T, x, phase)
    om, sysd = _uniform(names, rho, T)
    d = sysd.dFdrho(sysd.initialize_profiles())
    mu = pb.mu_res(om, rho, T)
    np.testing.assert_allclose(d[:, 0], mu, rtol=1e-12)
    np.testing.assert_allclose(d, np.repeat(d[:, :1], d.shape[1], axis=1), rtol=1e-12)


def test_bulk_consistency_3d():
    rho = np.array([0.021e30 / pb.N_A])
    om, sysd = _uniform(["argon"], rho, 100.0, N=8, nd=3)
    d = sysd.dFdrho(sysd.initialize_profiles())
    np.testing.assert_allclose(d.reshape(1, -1)[:, 0], pb.mu_res(om, rho, 100.0), rtol=1e-12)


def test_kernel_moments():
    # omega_hat(0): int rho dz -> 2w, int rho z^2 dz -> 4 pi w^3 / 3 (weighted_densities.jl:54-66)
    om, sysd = _uniform(["methane"], [1000.0], 150.0, N=64)
    for (ftype, width), K in zip(sysd.fields, sysd.kernels):
        if ftype == fn.INT_DZ:
            assert K[0, 0].real == pytest.approx(2 * width[0], rel=1e-14)
        elif ftype == fn.INT_Z2DZ:
            assert K[0, 0].real == pytest.approx(4 * np.pi * width[0] ** 3 / 3, rel=1e-14)


@pytest.mark.parametrize("names", [["water", "octane"], ["water", "ethanol"]])
def test_complex_step_matches_finite_differences(names):
    """Complex-step dPhi/dn against central differences: one association pair (analytic)
    and water + ethanol (4 pairs, the iterated solve whose derivative is the implicit one)."""
    rng = np.random.default_rng(0)
    _, om = models(names)
    T = 298.15
    rho = np.array([0.4, 0.6]) * pb.density(om, 1e5, T, [0.4, 0.6])
    om, sysd = _uniform(names, rho, T, N=16)
    n = sysd.weighted_densities(sysd.initialize_profiles())
    n = n * (1 + 0.05 * rng.standard_normal(n.shape))
    d = sysd.hsd_red[:, None]
    n[:, 3] = 0.05 * n[:, 1] * d * rng.standard_normal(n[:, 3].shape)   # vector field, |xi| < 1
    g = sysd.dphi(n)
    for i in range(2):
        for a in range(sysd.NF):
            h = 1e-5 * np.maximum(np.abs(n[i, a]), 1e-3)   # smaller steps drown the vector fields in rounding
            up, dn = n.copy(), n.copy()
            up[i, a] += h
            dn[i, a] -= h
            fd = (sysd.phi(up) - sysd.phi(dn)) / (2 * h)
            np.testing.assert_allclose(g[i, a], fd, rtol=2e-6, atol=1e-8 * np.abs(g).max())


def test_package_thermo_matches_oracle_bulk():
    import cdft_b200.thermo as th
    for names, p, T, x in [(["methane"], 1e7, 150.0, [1.0]), (["water", "octane"], 1e5, 298.15, [0.5, 0.5]),
                           (["water", "ethanol"], 1e5, 298.15, [0.3, 0.7])]:
        pm, om = models(names)
        r1 = pm.molar_density(p, T, x)
        r2 = pb.density(om, p, T, x)
        assert r1 == pytest.approx(r2, rel=1e-10)
        rho = np.asarray(x) * r1
        np.testing.assert_allclose(pm.mu_res(rho, T), pb.mu_res(om, rho, T), rtol=1e-12)
        assert pm.pressure(rho, T) == pytest.approx(pb.pressure(om, rho, T), rel=1e-10)
