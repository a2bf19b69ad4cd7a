"""Spherical and cylindrical (QDHT) grids through the C ABI against the oracle's
restatement (oracle/radial.py).  The reference's radial path is CPU-only; its QDHT
comes from Hankel.jl, which is not vendored, so the oracle restates the published
transform and is pinned only by bulk consistency (test_oracle_radial.py)."""
import numpy as np
import pytest

import _systems as S

pytestmark = pytest.mark.gpu

T_M, P_M = 150.0, 1e7


def _pair(names, coord, ub_L, N, core=None, precision="fp64"):
    import cdft_b200 as cd
    from oracle import pcsaft_bulk as pb
    from oracle import radial as rd
    pm, om = S.models(names)
    if names == ["methane"]:
        rb = [pb.density(om, P_M, T_M, [1.0])]
        cond = (P_M, T_M)
    else:   # water-rich liquid of the water/octane LLE
        r1, _ = S._lle(tuple(names), 1e5, 298.15)
        rb = list(r1)
        cond = (1e5, 298.15)
    L = om.length_scale()
    make = cd.Uniform1DSphr if coord == "sphr" else cd.Uniform1DCyl
    st = make(cond, rb, [0.0, ub_L * L], N)
    fields = None if core is None else [cd.HardCore(core * om.sigma[0])]
    sp = cd.DFTSystem(pm, st, fields, cd.DFTOptions(precision))
    ost = rd.RadialStructure(cond, rb, ub_L * L, N, coord)
    so = rd.RadialDFTSystem(om, ost, vext=sp.vext)
    return sp, so


@pytest.mark.parametrize("coord,ub_L,N", [("sphr", 10.0, 151), ("cyl", 20.0, 101)])
def test_bulk_consistency_radial_gpu(coord, ub_L, N):
    import cdft_b200 as cd
    from oracle import pcsaft_bulk as pb
    sp, so = _pair(["methane"], coord, ub_L, N)
    d = cd.dFdrho_res(sp, cd.initialize_profiles(sp))
    mu = pb.mu_res(so.model, sp.structure.rho_bulk, T_M)[0]
    assert abs(d[0, 0] - mu) < 1e-5          # the reference's tolerance
    do = so.dFdrho(so.initialize_profiles())
    assert float(np.max(np.abs(d - do)) / np.max(np.abs(do))) < 1e-10


@pytest.mark.parametrize("names", [["methane"], ["water", "octane"]])
@pytest.mark.parametrize("coord", ["sphr", "cyl"])
def test_functional_derivative_radial(coord, names):
    import cdft_b200 as cd
    sp, so = _pair(names, coord, 10.0, 121)
    rng = np.random.default_rng(3)
    rho = S.random_smooth_profile(sp, rng, amp=0.2)
    d = cd.dFdrho_res(sp, rho)
    do = so.dFdrho(rho)
    assert float(np.max(np.abs(d - do)) / np.max(np.abs(do))) < 1e-10
    assert cd.F_res(sp, rho) == pytest.approx(so.F_res(rho), rel=1e-11)


@pytest.mark.parametrize("coord,N", [("sphr", 151), ("cyl", 101)])
def test_converge_radial_hard_core(coord, N):
    """Methane around a hard core of radius 1.5 sigma at the origin, converged to 1e-11:
    fluid profiles agree with the oracle's to 1e-9."""
    import cdft_b200 as cd
    sp, so = _pair(["methane"], coord, 10.0, N, core=1.5)
    r0 = cd.initialize_profiles(sp)
    rho = r0.copy()
    kw = dict(beta=0.05, tol=1e-11, anderson_m=5, maxit=5000)
    res = cd.converge(sp, rho, **kw)
    ro, out = so.converge(r0.copy(), **kw)
    assert res.errcode == 0 and out.errcode == 0
    fluid = sp.vext[0] == 0
    assert float(np.max(np.abs(rho[0, fluid] / ro[0, fluid] - 1))) < 1e-9
    assert cd.free_energy(sp, rho) == pytest.approx(so.free_energy(ro), rel=1e-10)


def test_radial_runs_on_the_grid_engine():
    import cdft_b200 as cd
    from cdft_b200._lib import CDFTError
    sp, _ = _pair(["methane"], "sphr", 10.0, 101, core=1.5)
    rho = cd.initialize_profiles(sp)
    with pytest.raises(CDFTError):
        cd.converge(sp, rho, beta=0.05, tol=1e-8, engine="persistent")
    assert cd.converge(sp, rho, beta=0.05, tol=1e-8, engine="auto").errcode == 0


@pytest.mark.parametrize("coord,lb_L", [("sphr", 0.0), ("cyl", 2.0)])
def test_converge_radial_steele_wall(coord, lb_L):
    """A curved Steele wall (steele.jl:111-143): methane inside a spherical graphite pore
    (lb = 0, wall at ub) and around a graphite rod (lb > 0), converged on the grid engine
    with the clamped V_ext of the package; the oracle's RadialDFTSystem, given the Steele
    wall itself, reaches the same fixed point."""
    import cdft_b200 as cd
    from oracle import functional as fn, pcsaft_bulk as pb
    from oracle import radial as rd
    pm, om = S.models(["methane"])
    rb = [pb.density(om, P_M, T_M, [1.0])]
    L = om.length_scale()
    lb, ub, N = lb_L * L, 10.0 * L, 121
    make = cd.Uniform1DSphr if coord == "sphr" else cd.Uniform1DCyl
    sp = cd.DFTSystem(pm, make((P_M, T_M), rb, [lb, ub], N), cd.Steele(["graphite"]))
    so = rd.RadialDFTSystem(om, rd.RadialStructure((P_M, T_M), rb, ub, N, coord, lb=lb),
                            walls=[fn.SteeleWall.graphite()])
    np.testing.assert_allclose(sp.vext, so.vext, rtol=1e-12)
    rho = cd.initialize_profiles(sp)
    r0 = rho.copy()
    kw = dict(beta=0.1, tol=1e-12, anderson_m=5, maxit=5000)
    res = cd.converge(sp, rho, engine="grid", **kw)
    ro, out = so.converge(r0, **kw)
    assert res.errcode == 0 and out.errcode == 0, (res, out.errcode)
    assert float(np.max(np.abs(rho / ro - 1))) < 1e-8


def _sphere_pores(cases):
    """Methane in spherical graphite pores: (radius / L, N, pressure) per state point."""
    import cdft_b200 as cd
    from oracle import pcsaft_bulk as pb
    pm, om = S.models(["methane"])
    L = om.length_scale()
    out = []
    for ub_L, N, p in cases:
        rb = [pb.density(om, p, T_M, [1.0])]
        st = cd.Uniform1DSphr((p, T_M), rb, [0.0, ub_L * L], N)
        out.append(cd.DFTSystem(pm, st, cd.Steele(["graphite"])))
    return out


def test_radial_batch_equals_individual_bitwise():
    """Pores of one radius share one operator buffer and form column tiles of up to 8
    state points of the FP64 tensor-core GEMM (dense_group_kernel).  Radii with 5, 9 and 2
    pressures make tiles of 5, 8 + 1 and 2; every state point converged inside the batch
    gives the same bits and evaluation count as converged alone."""
    import cdft_b200 as cd
    assert cd.tuning("radial_dmma") in (1, 2)   # the tensor-core GEMM
    cases = ([(6.0, 101, p) for p in np.logspace(5, 7, 5)] + [(8.0, 131, p) for p in np.logspace(5, 7, 9)]
             + [(10.0, 151, p) for p in (2e6, 9e6)])
    systems = _sphere_pores(cases)
    rhos = [cd.initialize_profiles(sp) for sp in systems]
    kw = dict(beta=0.1, tol=1e-10, anderson_m=5, maxit=5000, engine="grid")
    singles = []
    for sp, r in zip(systems, rhos):
        rr = r.copy()
        singles.append((rr, cd.converge(sp, rr, **kw)))
    batch = [r.copy() for r in rhos]
    results = cd.batch_converge(systems, batch, **kw)
    for (rr, rs), rb, res in zip(singles, batch, results):
        assert res.errcode == rs.errcode == 0
        assert res.evaluations == rs.evaluations
        assert np.array_equal(rr, rb)
    for sp in systems:
        sp.close()


def test_radial_dmma_matches_warp_rows():
    """The tensor-core GEMM (radial_dmma = 1) and the warp-per-row matrix-vector kernel
    (radial_dmma = 0) apply the same operators in different summation orders: dF/drho
    agrees to 1e-13 of its scale at a random profile, and converged profiles to 1e-9."""
    import cdft_b200 as cd
    systems = _sphere_pores([(8.0, 131, 1e6), (8.0, 131, 5e6), (10.0, 151, 1e7)])
    kw = dict(beta=0.1, tol=1e-11, anderson_m=5, maxit=5000, engine="grid")
    got = {}
    default = cd.tuning("radial_dmma")
    try:
        for mode in (1, 0):
            cd.tuning("radial_dmma", mode)
            rho = S.random_smooth_profile(systems[0], np.random.default_rng(11), amp=0.2)
            d = cd.dFdrho_res(systems[0], rho)
            conv = [cd.initialize_profiles(sp) for sp in systems]
            res = cd.batch_converge(systems, conv, **kw)
            assert all(r.errcode == 0 for r in res)
            got[mode] = (d, conv)
    finally:
        cd.tuning("radial_dmma", default)
    d1, c1 = got[1]
    d0, c0 = got[0]
    assert float(np.max(np.abs(d1 - d0)) / np.max(np.abs(d0))) < 1e-13
    for a, b in zip(c1, c0):
        assert float(np.max(np.abs(a / b - 1))) < 1e-9
    for sp in systems:
        sp.close()


def test_radial_16_row_tiles_same_bits():
    """radial_dmma = 2 runs the GEMM with 16-row CTAs whose two row tiles share each input
    fragment; every output element takes the same products and additions in the same order
    as with 8-row CTAs (radial_dmma = 1): dF/drho and a batched converge agree bit for bit."""
    import cdft_b200 as cd
    systems = _sphere_pores([(8.0, 131, 1e6), (8.0, 131, 5e6), (10.0, 151, 1e7)])
    kw = dict(beta=0.1, tol=1e-10, anderson_m=5, maxit=5000, engine="grid")
    got = {}
    default = cd.tuning("radial_dmma")
    try:
        for mode in (1, 2):
            cd.tuning("radial_dmma", mode)
            rho = S.random_smooth_profile(systems[0], np.random.default_rng(5), amp=0.2)
            d = cd.dFdrho_res(systems[0], rho)
            conv = [cd.initialize_profiles(sp) for sp in systems]
            res = cd.batch_converge(systems, conv, **kw)
            got[mode] = (d, conv, [r.evaluations for r in res])
    finally:
        cd.tuning("radial_dmma", default)
    assert np.array_equal(got[1][0], got[2][0])
    assert got[1][2] == got[2][2]
    for a, b in zip(got[1][1], got[2][1]):
        assert np.array_equal(a, b)
    for sp in systems:
        sp.close()
