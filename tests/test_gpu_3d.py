"""3D periodic engine (FFT weighted densities) against the CPU oracle.

The configuration is a scaled-down version of the 3D benchmark case: PC-SAFT
argon at 100 K, rho_bulk = 0.021 A^-3, cubic periodic box with hard
spherical solutes (an external field the reference does not have; the oracle
receives the same V_ext array).  Tolerances as in the 1D parity tests."""
import functools

import numpy as np
import pytest

import _systems as S

pytestmark = pytest.mark.gpu

T_AR = 100.0


@functools.lru_cache(maxsize=None)
def _case(N=32, box_sigmas=8.0, nsol=2, precision="fp64"):
    import cdft_b200 as cd
    from oracle import functional as fn, pcsaft_bulk as pb
    pm, om = S.models(["argon"])
    rb = 0.021e30 / pb.N_A
    s = om.sigma[0]
    box = box_sigmas * s
    st = cd.Uniform3DCart((1e5, T_AR), [rb], [0.0, box], N)
    fields = None
    V = None
    if nsol:
        hs = cd.HardSphereSolutes(cd.HardSphereSolutes.seeded(nsol, 1.5 * s, box, 2 * box / N, seed=0), 1.5 * s)
        fields = [hs]
        V = hs.potential(pm, st)
    sp = cd.DFTSystem(pm, st, fields, cd.DFTOptions(precision))
    so = fn.DFTSystem(om, fn.Structure((1e5, T_AR), [rb], [(0.0, box)] * 3, (N, N, N)), vext=V)
    return sp, so


def test_bulk_consistency_3d_gpu():
    import cdft_b200 as cd
    from oracle import pcsaft_bulk as pb
    sp, so = _case(nsol=0)
    d = cd.dFdrho_res(sp, cd.initialize_profiles(sp))
    mu = pb.mu_res(so.model, sp.structure.rho_bulk, T_AR)
    np.testing.assert_allclose(d.reshape(1, -1), np.full((1, d.size), mu[0]), rtol=1e-11)


def test_phi_pointwise_3d():
    import cdft_b200 as cd
    rng = np.random.default_rng(11)
    sp, so = _case()
    rho = cd.initialize_profiles(sp) * (1 + 0.2 * rng.random(sp.structure.grid_shape))
    n = so.weighted_densities(rho).reshape(1, 9, -1)[:, :, ::97]
    f, g = cd.phi_pointwise(sp, n)
    osys = so
    nn = n.reshape(1, 9, -1)
    fo = osys.phi(nn)
    go = osys.dphi(nn)
    np.testing.assert_allclose(f, fo, rtol=1e-11, atol=1e-12 * np.max(np.abs(fo)))
    for a in range(9):
        scale = np.max(np.abs(go[0, a])) + 1e-300
        assert np.max(np.abs(g[0, a] - go[0, a])) <= 1e-10 * scale, a


def test_functional_derivative_3d():
    import cdft_b200 as cd
    rng = np.random.default_rng(12)
    sp, so = _case()
    N = sp.structure.ngrid[0]
    x = np.arange(N) / N
    smooth = (np.sin(2 * np.pi * x)[None, None, :] * np.cos(4 * np.pi * x)[None, :, None]
              + 0.5 * np.sin(2 * np.pi * x + 1.0)[:, None, None])
    rho = cd.initialize_profiles(sp) * (1 + 0.2 * smooth[None])
    d = cd.dFdrho_res(sp, rho)
    do = so.dFdrho(rho)
    assert float(np.max(np.abs(d - do)) / np.max(np.abs(do))) < 1e-10


def test_free_energy_3d():
    import cdft_b200 as cd
    sp, so = _case()
    rho = cd.initialize_profiles(sp)
    assert cd.F_res(sp, rho) == pytest.approx(so.F_res(rho), rel=1e-11)


def _fluid_solute_diff(sp, a, b):
    """(max relative difference over the fluid, max absolute difference inside the
    solutes / max density).  Inside a solute rho ~ exp(-100) rho_b: those values never
    enter the residual norm, so only their absolute size is controlled."""
    V = sp.vext
    fluid = a > 1e-12 * a.max() if V is None else V == 0
    rel = float(np.max(np.abs(a[fluid] / b[fluid] - 1)))
    ab = float(np.max(np.abs(a - b)[~fluid]) / a.max()) if (~fluid).any() else 0.0
    return rel, ab


def test_converge_3d_matches_oracle():
    """m = 10 as in the 3D configuration; converged to 1e-11 (the FFT path's FP64
    residual floor on this box sits near 1e-12 ||r0||), fluid profiles agree to 1e-9."""
    import cdft_b200 as cd
    sp, so = _case()
    rho = cd.initialize_profiles(sp)
    r0 = rho.copy()
    kw = dict(beta=0.1, tol=1e-11, anderson_m=10, maxit=1000)
    res = cd.converge(sp, rho, **kw)
    ro, out = so.converge(r0, **kw)
    assert res.errcode == 0 and out.errcode == 0
    rel, ab = _fluid_solute_diff(sp, rho, ro)
    assert rel < 1e-9 and ab < 1e-12, (rel, ab)
    assert cd.free_energy(sp, rho) == pytest.approx(so.free_energy(ro), rel=1e-10)


def test_converge_3d_mixed_reaches_fp64_fixed_point():
    import cdft_b200 as cd
    s64, _ = _case()
    s32, _ = _case(precision="mixed")
    r0 = cd.initialize_profiles(s64)
    a, b = r0.copy(), r0.copy()
    kw = dict(beta=0.1, tol=1e-10, anderson_m=10, maxit=1000)
    ra = cd.converge(s64, a, **kw)
    rb = cd.converge(s32, b, **kw)
    assert ra.errcode == 0 and rb.errcode == 0
    rel, ab = _fluid_solute_diff(s64, a, b)
    assert rel < 1e-7 and ab < 1e-10, (rel, ab)
    assert cd.free_energy(s32, b) == pytest.approx(cd.free_energy(s64, a), rel=1e-9)


@pytest.mark.parametrize("axis", [0, 1, 2])
def test_functional_derivative_3d_planar(axis):
    """Profiles varying along one axis only: the 3D operator must reduce to the 1D one."""
    import cdft_b200 as cd
    sp, so = _case(nsol=0)
    N = sp.structure.ngrid[0]
    x = np.arange(N) / N
    p1 = 1 + 0.2 * np.sin(2 * np.pi * x) + 0.1 * np.cos(6 * np.pi * x)
    shape = [1, 1, 1]
    shape[2 - axis] = N
    rho = cd.initialize_profiles(sp) * p1.reshape(shape)[None]
    d = cd.dFdrho_res(sp, rho)
    do = so.dFdrho(rho)
    assert float(np.max(np.abs(d - do)) / np.max(np.abs(do))) < 1e-10


@pytest.mark.parametrize("N", [64, 128])
def test_functional_derivative_3d_bench_box(N):
    """The 3D benchmark box itself (edge 16 sigma, 27 solutes) at 64^3 and 128^3."""
    import cdft_b200 as cd
    sp, so = _case(N=N, box_sigmas=16.0, nsol=27)
    x = np.arange(N) / N
    smooth = (np.sin(2 * np.pi * x)[None, None, :] * np.cos(4 * np.pi * x)[None, :, None]
              + 0.5 * np.sin(6 * np.pi * x + 1.0)[:, None, None])
    rho = cd.initialize_profiles(sp) * (1 + 0.2 * smooth[None])
    d = cd.dFdrho_res(sp, rho)
    do = so.dFdrho(rho)
    assert float(np.max(np.abs(d - do)) / np.max(np.abs(do))) < 1e-10


@pytest.mark.parametrize("axis", [0, 2])
def test_functional_derivative_256_planar_matches_1d(axis):
    """256^3 (the largest box): a profile varying along one axis gives the 1D engine's
    dF/drho on the same N points and period, in every plane."""
    import cdft_b200 as cd
    from oracle import pcsaft_bulk as pb
    N = 256
    pm, om = S.models(["argon"])
    rb = 0.021e30 / pb.N_A
    box = 16.0 * om.sigma[0]
    s3 = cd.DFTSystem(pm, cd.Uniform3DCart((1e5, T_AR), [rb], [0.0, box], N), None, cd.DFTOptions("fp64"))
    s1 = cd.DFTSystem(pm, cd.Uniform1DCart((1e5, T_AR), [rb], [0.0, box], N), None, cd.DFTOptions("fp64"))
    x = np.arange(N) / N
    p1 = 1 + 0.2 * np.sin(2 * np.pi * x) + 0.1 * np.cos(10 * np.pi * x)
    shape = [1, 1, 1]
    shape[2 - axis] = N
    rho3 = np.broadcast_to(rb * p1.reshape(shape), (N, N, N))[None].copy()
    d3 = cd.dFdrho_res(s3, rho3)
    d1 = cd.dFdrho_res(s1, (rb * p1)[None].copy())
    ref = np.broadcast_to(d1[0].reshape(shape), (N, N, N))
    assert float(np.max(np.abs(d3[0] - ref)) / np.max(np.abs(d1))) < 1e-11


def test_converge_256_mixed_matches_fp64():
    """The 3D benchmark box at 256^3 (27 solutes, m = 10, tol 1e-10): the mixed run
    reaches the FP64 fixed point.  At this size FP32 FFT noise inside the solutes rounds
    to exactly 0.0 at some points in some evaluations; the functional has to stay finite
    there, or one evaluation's NaN sends the liquid to another fixed point."""
    import cdft_b200 as cd
    from oracle import pcsaft_bulk as pb
    N = 256
    pm, om = S.models(["argon"])
    s = om.sigma[0]
    box = 16.0 * s
    rb = 0.021e30 / pb.N_A
    hs = cd.HardSphereSolutes(cd.HardSphereSolutes.seeded(27, 1.5 * s, box, 2 * box / N, seed=0), 1.5 * s)
    out = {}
    for prec in ("fp64", "mixed"):
        sp = cd.DFTSystem(pm, cd.Uniform3DCart((1e5, T_AR), [rb], [0.0, box], N), [hs], cd.DFTOptions(prec))
        rho = cd.initialize_profiles(sp)
        res = cd.converge(sp, rho, beta=0.1, tol=1e-10, anderson_m=10, maxit=2000, engine="grid")
        assert res.errcode == 0, (prec, res)
        out[prec] = (sp, rho, cd.free_energy(sp, rho))
    (s64, a, fa), (s32, b, fb) = out["fp64"], out["mixed"]
    rel, ab = _fluid_solute_diff(s64, a, b)
    assert rel < 1e-6 and ab < 1e-10, (rel, ab)
    assert fb == pytest.approx(fa, rel=1e-9)
    s64.close()
    s32.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("N", [32, 64, 128])
def test_tma_and_fused_passes_equal_plain_kernels(N, precision):
    """The TMA tile kernels of the y/z passes and the fused x pass (inverse x-FFT, Phi,
    forward x-FFT in one kernel) compute each line and each point with the arithmetic of
    the per-stage kernels."""
    import cdft_b200 as cd
    sp, _ = _case(N=N, box_sigmas=8.0 if N == 32 else 16.0, nsol=2 if N == 32 else 27, precision=precision)
    x = np.arange(N) / N
    smooth = (np.sin(2 * np.pi * x)[None, None, :] * np.cos(4 * np.pi * x)[None, :, None]
              + 0.5 * np.sin(6 * np.pi * x + 1.0)[:, None, None])
    rho = cd.initialize_profiles(sp) * (1 + 0.2 * smooth[None])
    out = {}
    try:
        for tma, fused in ((0, 0), (1, 0), (1, 1)):
            cd.tuning("fft3d_tma", tma)
            cd.tuning("fft3d_fused_phi", fused)
            out[(tma, fused)] = cd.dFdrho_res(sp, rho)
    finally:
        cd.tuning("fft3d_tma", 1)
        cd.tuning("fft3d_fused_phi", 1)
    ref = out[(0, 0)]
    # the TMA passes: the same arithmetic, to the last bit
    assert np.array_equal(out[(1, 0)], ref)
    # the fused x pass evaluates Phi on two threads per point (the hard-sphere/association
    # and chain/dispersion halves of the same sweep): equal to rounding
    assert float(np.max(np.abs(out[(1, 1)] - ref)) / np.max(np.abs(ref))) < 1e-14
