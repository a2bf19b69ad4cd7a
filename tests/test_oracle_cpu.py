"""The C++ restatement of converge! (oracle/cpu_converge.cpp, the timed CPU baseline)
against the NumPy oracle (CPU only)."""
import numpy as np
import pytest

from golden import make_fixtures as mf
from oracle import cpu, functional as fn, pcsaft_bulk as pb


@pytest.fixture(scope="module", autouse=True)
def _built():
    cpu.build()


def _methane_wall():
    om = mf.oracle_model(["methane"])
    T, p, N = 150.0, 1e7, 201
    rb = pb.density(om, p, T, [1.0])
    s = om.sigma[0]
    return fn.DFTSystem(om, fn.Structure((p, T), [rb], [(0.5 * s, 4.5 * s)], (N,)), [fn.SteeleWall.graphite()])


def _water_octane(N=300):
    om = mf.oracle_model(["water", "octane"])
    T, p = 298.15, 1e5
    x1, x2 = pb.lle_binary(om, p, T)
    r1 = pb.density(om, p, T, x1) * x1
    r2 = pb.density(om, p, T, x2) * x2
    s = om.sigma[0]
    return fn.DFTSystem(om, fn.Structure((p, T), list(r1), [(-30 * s, 30 * s)], (N,), kind="twophase",
                                         rho_bulk2=list(r2)))


@pytest.mark.parametrize("case", ["methane_wall", "water_octane"])
def test_functional_derivative_matches_numpy_oracle(case):
    so = _methane_wall() if case == "methane_wall" else _water_octane()
    rho = so.initialize_profiles()
    with np.errstate(all="ignore"):
        a = so.dFdrho(rho)
    b = cpu.functional_derivative(so, rho)
    for i in range(so.nc):
        assert np.max(np.abs(a[i] - b[i])) <= 1e-11 * np.max(np.abs(a[i]))


def test_converge_matches_numpy_oracle_trajectory():
    """Same aasol: the same number of evaluations and the same fixed point."""
    so = _methane_wall()
    rho0 = so.initialize_profiles()
    with np.errstate(all="ignore"):
        ro, out = so.converge(rho0.copy(), beta=0.1, tol=1e-13, anderson_m=5)
    r = [rho0.copy()]
    res, hist = cpu.batch_converge([so], r, nthreads=1, history_cap=200, beta=0.1, tol=1e-13, anderson_m=5)
    assert res[0].errcode == 0 and res[0].evaluations == len(out.history)
    np.testing.assert_allclose(hist[0][:20], out.history[:20], rtol=1e-9)
    assert float(np.max(np.abs(r[0] / ro - 1))) < 1e-11


def test_batch_threads_give_identical_results():
    om = mf.oracle_model(["methane"])
    s = om.sigma[0]
    systems = []
    specs = mf.isotherm_specs()
    for H, p, N in (specs[0], specs[27], specs[63]):
        rb = mf.stable_bulk_density(om, p, 150.0)
        systems.append(fn.DFTSystem(om, fn.Structure((p, 150.0), [rb], [(0.7 * s, H - 0.7 * s)], (N,)),
                                    [fn.SteeleWall.graphite(H)]))
    r1 = [so.initialize_profiles() for so in systems]
    r4 = [x.copy() for x in r1]
    a, _ = cpu.batch_converge(systems, r1, nthreads=1, beta=0.1, tol=1e-10, anderson_m=5)
    b, _ = cpu.batch_converge(systems, r4, nthreads=3, beta=0.1, tol=1e-10, anderson_m=5)
    for x, y, u, v in zip(a, b, r1, r4):
        assert x.errcode == y.errcode == 0 and x.evaluations == y.evaluations
        assert np.array_equal(u, v)
