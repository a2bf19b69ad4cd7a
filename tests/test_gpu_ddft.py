"""The DDFT right-hand side through the C ABI against the oracle's restatement of
ddft_rhs_log! (ext/SciMLBasecDFTExt.jl:10-61): FFT maps in the oracle, per-axis
circulants on the device.  1D with a wall and with two components, 3D on the solute box;
and at a converged interface the right-hand side vanishes (a fixed point of converge! is a
steady state of DDFT)."""
import numpy as np
import pytest

import _systems as S

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


@pytest.mark.parametrize("case", ["methane_wall", "water_octane"])
def test_ddft_rhs_1d_matches_oracle(case):
    import cdft_b200 as cd
    rng = np.random.default_rng(21)
    if case == "methane_wall":
        sp, so = S.methane_wall(N=201)
        rho = cd.initialize_profiles(sp)
    else:
        sp, so = S.water_octane_lle(N=256)
        rho = S.random_smooth_profile(sp, rng)
    eta = np.log(rho)
    d = cd.ddft_rhs(sp, eta)
    do = so.ddft_rhs(eta)
    for i in range(sp.nc):
        assert _rel(d[i], do[i]) < 1e-10, (i, _rel(d[i], do[i]))


def test_ddft_rhs_3d_matches_oracle():
    import cdft_b200 as cd
    from oracle import functional as fn
    from golden import make_fixtures as mf
    N = 32
    pm, om = S.models(["argon"])
    s = om.sigma[0]
    box = 16 * s
    rb = 0.021e30 / cd.N_A
    centres = cd.HardSphereSolutes.seeded(27, 1.5 * s, box, 2 * box / 128, seed=0)
    sp = cd.DFTSystem(pm, cd.Uniform3DCart((1e5, 100.0), [rb], [0.0, box], N), cd.HardSphereSolutes(centres, 1.5 * s))
    so = fn.DFTSystem(om, fn.Structure((1e5, 100.0), [rb], [(0.0, box)] * 3, (N, N, N)),
                      vext=mf.solute_vext(N, box, centres, 1.5 * s))
    rng = np.random.default_rng(22)
    rho = cd.initialize_profiles(sp) * (1 + 0.02 * rng.standard_normal((1, N, N, N)))
    eta = np.log(rho)
    d = cd.ddft_rhs(sp, eta)
    do = so.ddft_rhs(eta)
    assert _rel(d, do) < 1e-10
    sp.close()


def test_ddft_rhs_vanishes_at_a_converged_interface():
    import cdft_b200 as cd
    sp, _ = S.octane_vle(N=256)
    rho = cd.initialize_profiles(sp)
    scale = np.max(np.abs(cd.ddft_rhs(sp, np.log(rho))))
    res = cd.converge(sp, rho, beta=0.01, tol=1e-12, anderson_m=5, maxit=20000)
    assert res.errcode == 0
    f, u0, _ = cd.ddft_problem(sp, rho, (0.0, 1.0))
    assert np.max(np.abs(f(u0))) < 1e-8 * scale
