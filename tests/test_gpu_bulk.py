"""Batched bulk densities on the device (cdft_bulk_density) against the host bulk
PC-SAFT (cdft_b200.thermo, itself pinned to the oracle's bulk equations): the stable
root of every isotherm state point, liquid and vapour roots of n-octane and water
(2B association), and a water + n-octane liquid.  Roots to 1e-12 relative."""
import numpy as np
import pytest

import _systems as S

pytestmark = pytest.mark.gpu


def test_isotherm_stable_densities():
    import bench
    import cdft_b200 as cd
    model = cd.PCSAFT(["methane"], **bench.METHANE)
    ps = np.array([p for _, p, _ in bench.isotherm_specs()])
    got = cd.bulk_density(model, ps, bench.T_ISO, [1.0])
    want = np.array([model.stable_density(p, bench.T_ISO, [1.0]) for p in ps])
    np.testing.assert_allclose(got, want, rtol=1e-12)


@pytest.mark.parametrize("names,T,x", [(["octane"], 298.15, [1.0]), (["water"], 298.15, [1.0]),
                                       (["water", "octane"], 298.15, [0.3, 0.7])])
def test_liquid_and_vapour_roots(names, T, x):
    import cdft_b200 as cd
    pm, _ = S.models(names)
    ps = np.logspace(2, 6, 9)
    for phase in ("liquid", "vapour", "stable"):
        try:
            want = np.array([pm.molar_density(p, T, x, phase) if phase != "stable" else pm.stable_density(p, T, x)
                             for p in ps])
        except ValueError:
            continue
        got = cd.bulk_density(pm, ps, T, x, phase)
        np.testing.assert_allclose(got, want, rtol=1e-12, err_msg=phase)


def test_cross_association_is_refused():
    import cdft_b200 as cd
    from cdft_b200._lib import CDFTError
    pm, _ = S.models(["water", "ethanol"])
    with pytest.raises(CDFTError):
        cd.bulk_density(pm, [1e5], 298.15, [0.5, 0.5], "liquid")


@pytest.mark.parametrize("name,Ts", [("octane", [250.0, 298.15, 350.0, 450.0, 500.0]),
                                     ("methane", [100.0, 120.0, 150.0, 170.0]),
                                     ("water", [298.15, 373.15, 450.0])])
def test_saturation_matches_oracle(name, Ts):
    """Pure-component coexistence of every temperature in one launch (cdft_saturation_pure)
    against the oracle's saturation_pure (the same equations p_l = p_v, mu_l = mu_v from the
    same starting point, Newton with a finite-difference Jacobian on the host): both
    densities and the pressure of the vapour root to 1e-10, water with its 2B association.
    (The oracle reports the liquid root's pressure, whose compressibility factor is ~5e-6
    for octane at 250 K: the last bits of rho_l move it by ~1e-7.)"""
    import cdft_b200 as cd
    from oracle import pcsaft_bulk as pb
    pm, om = S.models([name])
    p, rl, rv = cd.saturation(pm, Ts)
    for k, T in enumerate(Ts):
        _, wl, wv = pb.saturation_pure(om, T)
        wp = pb.pressure(om, [wv], T)
        np.testing.assert_allclose([p[k], rl[k], rv[k]], [wp, wl, wv], rtol=1e-10, err_msg=f"{name} {T} K")
        assert rl[k] > rv[k]


def test_saturation_above_the_critical_temperature_is_refused():
    """Above T_c the Newton iteration collapses onto one phase: status 3, a ValueError."""
    import cdft_b200 as cd
    pm, _ = S.models(["methane"])
    with pytest.raises(ValueError):
        cd.saturation(pm, [120.0, 260.0])


def test_surface_tension_of_a_model():
    """surface_tension(model, T) (surface_tension.jl:13-29) for n-octane at three
    temperatures: the device coexistence, one batched converge of the 201-point
    TwoPhase1DCart systems on [-10L, 10L] and gamma = surface_tension(system, rho) / 2.  It
    equals the same construction from the oracle's coexistence converged one system at a
    time (1e-7), is a float for a scalar T, and falls with T."""
    import cdft_b200 as cd
    from oracle import pcsaft_bulk as pb
    pm, om = S.models(["octane"])
    Ts = [280.0, 298.15, 320.0]
    g = cd.surface_tension(pm, Ts)
    L = pm.length_scale()
    for k, T in enumerate(Ts):
        _, wl, wv = pb.saturation_pure(om, T)
        wp = pb.pressure(om, [wv], T)
        sy = cd.DFTSystem(pm, cd.TwoPhase1DCart((wp, T), [wl], [wv], [-10 * L, 10 * L], 201))
        rho = cd.initialize_profiles(sy)
        cd.converge(sy, rho)
        want = cd.surface_tension(sy, rho) / 2
        sy.close()
        assert g[k] == pytest.approx(want, rel=1e-7), T
    assert g[0] > g[1] > g[2] > 0.0
    assert 0.005 < g[1] < 0.05   # J/m^2: n-octane's tension at 298 K is about 0.021
    assert isinstance(cd.surface_tension(pm, 298.15), float)
