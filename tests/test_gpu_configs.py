"""GPU parity at the benchmark configurations' own sizes, against committed oracle
fixtures (``tests/golden/*.npz``, written by ``tests/golden/make_fixtures.py``).

Each test builds the package system from the inputs stored in the fixture (bulk
densities of the oracle's bulk solves, bounds, grid), converges it through the C ABI
to a tolerance below the 1e-9 parity floor (the reference's stopping test is on the
damped residual of ln rho, so a 1e-10 run sits near 1e-9 in rho), and compares:

* FP64: profiles within 1e-9 relative, gamma / Omega_ex / adsorption within 1e-9;
* mixed (FP32 convolutions and Phi, FP64 solver): |dgamma/gamma| and
  |dOmega/Omega| within 1e-6 of the FP64 oracle.

Two-interface boxes (c2, c4) are compared after removing the interfaces' zero
modes (see ``_systems.aligned_log_diff``)."""
import functools
import os

import numpy as np
import pytest

import _systems as S

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
RHO_TOL = 1e-9      # FP64 parity bar in rho
GAMMA_TOL = 1e-9    # FP64 parity bar in gamma
MIXED_TOL = 1e-6    # mixed path: |dgamma/gamma| against the FP64 oracle


@functools.lru_cache(maxsize=None)
def fixture(name):
    path = os.path.join(GOLDEN, name + ".npz")
    if not os.path.exists(path):
        pytest.fail(f"fixture {name}.npz is missing: run tests/golden/make_fixtures.py")
    with np.load(path) as z:
        return {k: z[k] for k in z.files}


def _pkg_model(names):
    pm, _ = S.models(names)
    return pm


def _c1_system(precision):
    import cdft_b200 as cd
    f = fixture("c1_methane_wall_201")
    st = cd.Uniform1DCart((float(f["p"]), float(f["T"])), list(f["rho_bulk"]), list(f["bounds"]), int(f["N"]))
    return cd.DFTSystem(_pkg_model(["methane"]), st, cd.Steele(["graphite"]), cd.DFTOptions(precision)), f


def _interface_system(name, names, precision):
    import cdft_b200 as cd
    f = fixture(name)
    st = cd.TwoPhase1DCart((float(f["p"]), float(f["T"])), list(f["rho_bulk"]), list(f["rho_bulk2"]),
                           list(f["bounds"]), int(f["N"]))
    return cd.DFTSystem(_pkg_model(names), st, None, cd.DFTOptions(precision)), f


@pytest.mark.parametrize("engine", ["grid", "persistent"])
def test_c1_methane_wall(engine):
    import cdft_b200 as cd
    sp, f = _c1_system("fp64")
    rho = cd.initialize_profiles(sp)
    res = cd.converge(sp, rho, beta=0.1, tol=1e-13, anderson_m=5, engine=engine)
    assert res.errcode == 0, res
    assert float(np.max(np.abs(rho / f["rho"] - 1))) < RHO_TOL
    assert cd.surface_tension(sp, rho) == pytest.approx(float(f["omega_ex"]), rel=GAMMA_TOL)
    assert cd.adsorption(sp, rho)[0] == pytest.approx(float(f["adsorption"][0]), rel=GAMMA_TOL)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_c2_octane_vle_2048(precision):
    """n-octane vapour-liquid interface, 2048 points over 40 sigma: rho and gamma."""
    import cdft_b200 as cd
    sp, f = _interface_system("c2_octane_vle_2048", ["octane"], precision)
    rho = cd.initialize_profiles(sp)
    res = cd.converge(sp, rho, beta=0.01, tol=1e-13, anderson_m=5, maxit=20000)
    assert res.errcode == 0, res
    g = cd.surface_tension(sp, rho) / 2
    err, shifts = S.aligned_log_diff(rho, f["rho"])
    if precision == "fp64":
        assert err < RHO_TOL, (err, shifts)
        assert g == pytest.approx(float(f["gamma"]), rel=GAMMA_TOL)
    else:
        assert abs(g / float(f["gamma"]) - 1) < MIXED_TOL
    # the interfaces sit within a small fraction of a grid cell of the oracle's; the FP32 phase
    # of a mixed run drifts along the zero modes (no restoring force), which the FP64 polish
    # keeps, so its bound is looser
    assert max(abs(x) for x in shifts) < (1e-3 if precision == "fp64" else 2e-2), shifts


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_c4_water_octane_lle_4096(precision):
    """Water (2B) + n-octane liquid-liquid interface, 4096 points over 60 sigma_water."""
    import cdft_b200 as cd
    sp, f = _interface_system("c4_water_octane_lle_4096", ["water", "octane"], precision)
    rho = cd.initialize_profiles(sp)
    res = cd.converge(sp, rho, beta=0.01, tol=1e-12, anderson_m=5, maxit=40000)
    assert res.errcode == 0, res
    g = cd.surface_tension(sp, rho) / 2
    err, shifts = S.aligned_log_diff(rho, f["rho"])
    if precision == "fp64":
        assert err < RHO_TOL, (err, shifts)
        assert g == pytest.approx(float(f["gamma"]), rel=GAMMA_TOL)
    else:
        assert abs(g / float(f["gamma"]) - 1) < MIXED_TOL
    # the interfaces sit within a small fraction of a grid cell of the oracle's; the FP32 phase
    # of a mixed run drifts along the zero modes (no restoring force), which the FP64 polish
    # keeps, so its bound is looser
    assert max(abs(x) for x in shifts) < (1e-3 if precision == "fp64" else 2e-2), shifts


def _isotherm_systems(precision):
    import cdft_b200 as cd
    f = fixture("c3_isotherm64")
    pm = _pkg_model(["methane"])
    s = pm.sigma[0]
    systems = []
    for H, p, N, rb in zip(f["H"], f["p"], f["N"], f["rho_bulk"]):
        st = cd.Uniform1DCart((float(p), float(f["T"])), [float(rb)], [0.7 * s, float(H) - 0.7 * s], int(N))
        systems.append(cd.DFTSystem(pm, st, cd.Steele(["graphite"], float(H)), cd.DFTOptions(precision)))
    return systems, f


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_c3_isotherm_all_64_state_points(precision):
    """The headline workload: all 64 slit-pore state points converged in one batch
    (the persistent engine); every profile, adsorption and Omega_ex is compared."""
    import cdft_b200 as cd
    systems, f = _isotherm_systems(precision)
    rhos = [cd.initialize_profiles(sy) for sy in systems]
    results = cd.batch_converge(systems, rhos, beta=0.1, tol=1e-13, anderson_m=5)
    off = f["offsets"]
    worst = {"rho": 0.0, "adsorption": 0.0, "omega": 0.0}
    for k, (sy, r, res) in enumerate(zip(systems, rhos, results)):
        assert res.errcode == 0, (k, res)
        ref = f["rho"][off[k]:off[k + 1]]
        worst["rho"] = max(worst["rho"], float(np.max(np.abs(r[0] / ref - 1))))
        worst["adsorption"] = max(worst["adsorption"], abs(cd.adsorption(sy, r)[0] / f["adsorption"][k] - 1))
        worst["omega"] = max(worst["omega"], abs(cd.surface_tension(sy, r) / f["omega_ex"][k] - 1))
    for sy in systems:
        sy.close()
    if precision == "fp64":
        assert worst["rho"] < RHO_TOL and worst["adsorption"] < GAMMA_TOL and worst["omega"] < GAMMA_TOL, worst
    else:
        assert worst["adsorption"] < MIXED_TOL and worst["omega"] < MIXED_TOL, worst


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_c5_solutes_128(precision):
    """Argon around 27 hard solutes in the periodic 128^3 box (edge 16 sigma), m = 10,
    converged to 1e-11: the fluid profile (stored on every 4th point per axis) within
    1e-9 and Omega_ex within 1e-9 of the oracle (mixed: Omega_ex within 1e-6)."""
    import cdft_b200 as cd
    f = fixture("c5_solutes_128")
    N, st_ = int(f["N"]), int(f["stride"])
    pm = _pkg_model(["argon"])
    box = float(f["box"])
    st = cd.Uniform3DCart((float(f["p"]), float(f["T"])), list(f["rho_bulk"]), [0.0, box], N)
    hs = cd.HardSphereSolutes(f["centres"], float(f["radius"]))
    sp = cd.DFTSystem(pm, st, [hs], cd.DFTOptions(precision))
    rho = cd.initialize_profiles(sp)
    res = cd.converge(sp, rho, beta=0.1, tol=1e-11, anderson_m=10, maxit=1000, engine="grid")
    assert res.errcode == 0, res
    om = cd.surface_tension(sp, rho)
    fluid = sp.vext[0] == 0
    sub = (slice(None), slice(None, None, st_), slice(None, None, st_), slice(None, None, st_))
    fsub = fluid[sub[1:]]
    rel = float(np.max(np.abs(rho[sub][0][fsub] / f["rho_sub"][0][fsub] - 1)))
    sp.close()
    if precision == "fp64":
        assert rel < RHO_TOL, rel
        assert float(np.sum(rho[0][fluid])) == pytest.approx(float(f["fluid_sum"]), rel=1e-11)
        assert om == pytest.approx(float(f["omega_ex"]), rel=GAMMA_TOL)
    else:
        assert abs(om / float(f["omega_ex"]) - 1) < MIXED_TOL
