"""The general association path (several site pairs, assoc.jl:771-828) on the GPU against
the oracle: water + ethanol with self- and cross-association, 4 site pairs and 4 sites,
the reference's own water+ethanol case (test/test_models.jl:171-188).  Tolerances as the
one-pair parity tests: Phi and its gradient 1e-10, dF/drho 1e-10, bulk consistency 1e-11,
the converged profile 1e-9 against the committed oracle fixture."""
import os

import numpy as np
import pytest

import _systems as S

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _rel(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


def test_phi_pointwise_general_association():
    import cdft_b200 as cd
    rng = np.random.default_rng(11)
    sp, so = S.water_ethanol_wall(N=64)
    assert len(so.assoc_pairs) == 4
    rho = S.random_smooth_profile(sp, rng)
    n = so.weighted_densities(rho)
    n = n * (1 + 0.05 * rng.standard_normal(n.shape))
    f, g = cd.phi_pointwise(sp, n)
    fo = so.phi(n)
    go = so.dphi(n)
    np.testing.assert_allclose(f, fo, rtol=1e-11, atol=1e-12 * np.max(np.abs(fo)))
    for i in range(sp.nc):
        for a in range(so.NF):
            scale = np.max(np.abs(go[i, a])) + 1e-300
            assert np.max(np.abs(g[i, a] - go[i, a])) <= 1e-10 * scale, (i, a)


def test_functional_derivative_general_association():
    import cdft_b200 as cd
    rng = np.random.default_rng(12)
    sp, so = S.water_ethanol_wall(N=150)
    for rho in (cd.initialize_profiles(sp), S.random_smooth_profile(sp, rng)):
        d = cd.dFdrho_res(sp, rho)
        do = so.dFdrho(rho)
        for i in range(sp.nc):
            assert _rel(d[i], do[i]) < 1e-10, (i, _rel(d[i], do[i]))


def test_bulk_consistency_general_association():
    import cdft_b200 as cd
    pm, om = S.models(["water", "ethanol"])
    for x in ([0.5, 0.5], [0.9, 0.1], [0.2, 0.8]):
        x = np.asarray(x)
        rho_b = x * pm.molar_density(1e5, 298.15, x)
        L = om.length_scale()
        sysp = cd.DFTSystem(pm, cd.Uniform1DCart((1e5, 298.15), rho_b, [-10 * L, 10 * L], 3))
        d = cd.dFdrho_res(sysp, cd.initialize_profiles(sysp))
        np.testing.assert_allclose(d[:, 0], pm.mu_res(rho_b, 298.15), rtol=1e-11)
        sysp.close()


@pytest.mark.parametrize("engine", ["grid", "persistent"])
def test_converge_general_association_matches_fixture(engine):
    import cdft_b200 as cd
    fx = np.load(os.path.join(GOLDEN, "a9_water_ethanol_wall_150.npz"))
    sp, _ = S.water_ethanol_wall(N=int(fx["N"]))
    np.testing.assert_allclose(sp.structure.rho_bulk, fx["rho_bulk"], rtol=1e-12)
    rho = cd.initialize_profiles(sp)
    res = cd.converge(sp, rho, beta=0.01, tol=1e-12, anderson_m=5, maxit=10000, engine=engine)
    assert res.errcode == 0 and int(fx["errcode"]) == 0
    assert float(np.max(np.abs(rho / fx["rho"] - 1))) < 1e-9
    np.testing.assert_allclose(cd.adsorption(sp, rho), fx["adsorption"], rtol=1e-9)


def test_parameter_gradient_refuses_several_pairs():
    import cdft_b200 as cd
    from cdft_b200._lib import CDFTError
    sp, _ = S.water_ethanol_wall(N=64)
    with pytest.raises(CDFTError):
        cd.F_res_grad(sp, cd.initialize_profiles(sp))
