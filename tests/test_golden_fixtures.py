"""The committed oracle fixtures of the benchmark configurations (CPU).

Each stored converged profile must be a fixed point of the oracle's Picard map
ln rho -> ln G(rho) (GFix!, src/methods/converge.jl:235-242) to the residual its
stopping test allowed, and the stored gamma / adsorption must follow from it."""
import os

import numpy as np
import pytest

from golden import make_fixtures as mf

GOLDEN = os.path.dirname(os.path.abspath(mf.__file__))


def _load(name):
    path = os.path.join(GOLDEN, name + ".npz")
    if not os.path.exists(path):
        pytest.fail(f"fixture {name}.npz is missing: run tests/golden/make_fixtures.py")
    with np.load(path) as z:
        return {k: z[k] for k in z.files}


def _fixed_point_residual(so, rho, beta):
    """||beta (ln G(rho) - ln rho)||_2 / ||ln rho||_2 (the damped residual of aasol)."""
    with np.errstate(all="ignore"):
        lnG = so.get_new_profile(rho)
    x = np.log(rho)
    return float(np.linalg.norm(beta * (lnG - x)) / np.linalg.norm(x))


def test_c1_fixture_is_oracle_fixed_point():
    from oracle import functional as fn
    f = _load("c1_methane_wall_201")
    om = mf.oracle_model(["methane"])
    so = fn.DFTSystem(om, fn.Structure((float(f["p"]), float(f["T"])), list(f["rho_bulk"]), [tuple(f["bounds"])],
                                       (int(f["N"]),)), [fn.SteeleWall.graphite()])
    assert int(f["errcode"]) == 0
    assert _fixed_point_residual(so, f["rho"], 0.1) < 1e-13
    assert so.surface_tension(f["rho"]) == pytest.approx(float(f["omega_ex"]), rel=1e-13)


def test_c2_fixture_is_oracle_fixed_point():
    from oracle import functional as fn
    f = _load("c2_octane_vle_2048")
    om = mf.oracle_model(["octane"])
    st = fn.Structure((float(f["p"]), float(f["T"])), list(f["rho_bulk"]), [tuple(f["bounds"])], (int(f["N"]),),
                      kind="twophase", rho_bulk2=list(f["rho_bulk2"]))
    so = fn.DFTSystem(om, st)
    assert int(f["errcode"]) == 0 and int(f["N"]) == 2048
    assert _fixed_point_residual(so, f["rho"], 0.01) < 1e-13
    assert so.surface_tension(f["rho"]) / 2 == pytest.approx(float(f["gamma"]), rel=1e-13)
    assert float(f["gamma"]) > 0


def test_c3_fixture_covers_the_isotherm():
    from oracle import functional as fn
    f = _load("c3_isotherm64")
    specs = mf.isotherm_specs()
    assert len(f["H"]) == 64 and np.all(f["errcode"] == 0)
    assert [(float(H), float(p), int(N)) for H, p, N in zip(f["H"], f["p"], f["N"])] == specs
    om = mf.oracle_model(["methane"])
    s = om.sigma[0]
    off = f["offsets"]
    for k in (0, 27, 63):   # three state points: smallest, middle, largest pore
        H, p, N = specs[k]
        so = fn.DFTSystem(om, fn.Structure((p, float(f["T"])), [float(f["rho_bulk"][k])], [(0.7 * s, H - 0.7 * s)],
                                           (N,)), [fn.SteeleWall.graphite(H)])
        rho = f["rho"][off[k]:off[k + 1]][None]
        assert _fixed_point_residual(so, rho, 0.1) < 1e-13
        assert so.adsorption(rho)[0] == pytest.approx(float(f["adsorption"][k]), rel=1e-13)


def test_c4_fixture_is_a_converged_interface():
    """c4 comes from the oracle's C++ restatement (the NumPy run takes hours at 4096 points):
    its stored profile must be a fixed point of the NumPy oracle's map as well."""
    from oracle import functional as fn
    f = _load("c4_water_octane_lle_4096")
    assert int(f["errcode"]) == 0 and int(f["N"]) == 4096 and f["rho"].shape == (2, 4096)
    assert float(f["gamma"]) > 0
    om = mf.oracle_model(["water", "octane"])
    st = fn.Structure((float(f["p"]), float(f["T"])), list(f["rho_bulk"]), [tuple(f["bounds"])], (int(f["N"]),),
                      kind="twophase", rho_bulk2=list(f["rho_bulk2"]))
    so = fn.DFTSystem(om, st)
    assert _fixed_point_residual(so, f["rho"], 0.01) < 1e-12
    assert so.surface_tension(f["rho"]) / 2 == pytest.approx(float(f["gamma"]), rel=1e-12)


def test_c5_fixture_present():
    g = _load("c5_solutes_128")
    assert int(g["errcode"]) == 0 and int(g["N"]) == 128 and g["rho_sub"].shape == (1, 32, 32, 32)
    assert g["centres"].shape == (27, 3)


def test_white_bear_series_departure_recorded():
    """The oracle's series form of the White-Bear bracket near n3 = 0 against the
    reference's closed form: the recorded departure in every configuration."""
    f1 = _load("c1_methane_wall_201")
    f2 = _load("c2_octane_vle_2048")
    f3 = _load("c3_isotherm64")
    for f in (f1, f2):
        assert np.isfinite(float(f["closed_rho_rel_diff"]))
    assert f3["closed_rho_rel_diff"].shape == (64,)


def test_a9_fixture_is_oracle_fixed_point():
    """Water + ethanol at a graphite wall: the general association path (4 site pairs)."""
    from oracle import functional as fn
    f = _load("a9_water_ethanol_wall_150")
    om = mf.oracle_model(["water", "ethanol"])
    s = om.sigma[0]
    so = fn.DFTSystem(om, fn.Structure((float(f["p"]), float(f["T"])), list(f["rho_bulk"]), [(0.5 * s, 4.5 * s)],
                                       (int(f["N"]),)), [fn.SteeleWall.graphite()])
    assert len(so.assoc_pairs) == 4
    assert int(f["errcode"]) == 0
    assert _fixed_point_residual(so, f["rho"], 0.01) < 1e-12
    np.testing.assert_allclose(so.adsorption(f["rho"]), f["adsorption"], rtol=1e-13)
