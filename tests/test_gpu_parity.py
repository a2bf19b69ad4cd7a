"""GPU parity: the CUDA path (through the C ABI) against the CPU oracle on the
same seeded inputs.  Tolerances (FP64 path): Phi/gradients and dF/drho 1e-10
relative to the field's scale; converged profiles 1e-9 relative (the FP64
parity bar in rho), gamma 1e-9 relative."""
import numpy as np
import pytest

import _systems as S

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


_aligned_log_diff = S.aligned_log_diff


@pytest.mark.parametrize("case", ["methane", "water_octane", "octane"])
def test_phi_pointwise_matches_complex_step(case):
    import cdft_b200 as cd
    rng = np.random.default_rng(1)
    if case == "methane":
        sp, so = S.methane_wall(N=64)
    elif case == "octane":
        sp, so = S.octane_vle(N=64)
    else:
        sp, so = S.water_octane_lle(N=64)
    rho = S.random_smooth_profile(sp, rng)
    n = so.weighted_densities(rho)                    # (nc, NF, N)
    n = n * (1 + 0.05 * rng.standard_normal(n.shape))
    f, g = cd.phi_pointwise(sp, n)
    fo = so.phi(n)
    go = so.dphi(n)
    np.testing.assert_allclose(f, fo, rtol=1e-11, atol=1e-12 * np.max(np.abs(fo)))
    for i in range(sp.nc):
        for a in range(so.NF):
            scale = np.max(np.abs(go[i, a])) + 1e-300
            assert np.max(np.abs(g[i, a] - go[i, a])) <= 1e-10 * scale, (i, a)


@pytest.mark.parametrize("case", ["methane_wall", "slit", "octane", "water_octane"])
def test_functional_derivative_matches_oracle(case):
    import cdft_b200 as cd
    rng = np.random.default_rng(2)
    if case == "methane_wall":
        sp, so = S.methane_wall(N=201)
        rho = cd.initialize_profiles(sp)
    elif case == "slit":
        sp, so = S.slit_pore(3e-9, 1e5, N=150)
        rho = cd.initialize_profiles(sp)
    elif case == "octane":
        sp, so = S.octane_vle(N=256)
        rho = S.random_smooth_profile(sp, rng)
    else:
        sp, so = S.water_octane_lle(N=256)
        rho = S.random_smooth_profile(sp, rng)
    d = cd.dFdrho_res(sp, rho)
    do = so.dFdrho(rho)
    for i in range(sp.nc):
        assert _rel(d[i], do[i]) < 1e-10, (i, _rel(d[i], do[i]))


def test_bulk_consistency_on_gpu():
    import cdft_b200 as cd
    from oracle import pcsaft_bulk as pb
    for names, p, T, x in [(["methane"], 1e7, 150.0, [1.0]), (["water", "octane"], 1e5, 298.15, [0.5, 0.5])]:
        pm, om = S.models(names)
        x = np.asarray(x)
        rho_b = x * pb.density(om, p, T, x)
        L = om.length_scale()
        sysp = cd.DFTSystem(pm, cd.Uniform1DCart((p, T), rho_b, [-10 * L, 10 * L], 3))
        d = cd.dFdrho_res(sysp, cd.initialize_profiles(sysp))
        np.testing.assert_allclose(d[:, 0], pb.mu_res(om, rho_b, T), rtol=1e-11)


def test_free_energy_matches_oracle():
    import cdft_b200 as cd
    rng = np.random.default_rng(3)
    sp, so = S.water_octane_lle(N=128)
    rho = S.random_smooth_profile(sp, rng)
    assert cd.F_res(sp, rho) == pytest.approx(so.F_res(rho), rel=1e-11)


@pytest.mark.parametrize("engine", ["grid", "persistent"])
def test_converge_methane_wall_tight(engine):
    """Config-1 system (201 points, m=5, beta=0.1), converged to 1e-13: profiles agree to 1e-9."""
    import cdft_b200 as cd
    sp, so = S.methane_wall(N=201)
    rho = cd.initialize_profiles(sp)
    rho0 = rho.copy()
    res = cd.converge(sp, rho, beta=0.1, tol=1e-13, anderson_m=5, engine=engine)
    ro, out = so.converge(rho0, beta=0.1, tol=1e-13, anderson_m=5)
    assert res.idid and res.errcode == 0 and out.errcode == 0
    assert float(np.max(np.abs(rho / ro - 1))) < 1e-9
    assert cd.adsorption(sp, rho)[0] == pytest.approx(so.adsorption(ro)[0], rel=1e-9)


@pytest.mark.parametrize("engine", ["grid", "persistent"])
def test_converge_methane_wall_same_trajectory(engine):
    """At the configuration's own tolerance (1e-10) the GPU follows the oracle's
    aasol trajectory: same phases, same iteration count, same residual history."""
    import cdft_b200 as cd
    sp, so = S.methane_wall(N=201)
    rho = cd.initialize_profiles(sp)
    rho0 = rho.copy()
    res = cd.converge(sp, rho, beta=0.1, tol=1e-10, anderson_m=5, engine=engine)
    ro, out = so.converge(rho0, beta=0.1, tol=1e-10, anderson_m=5)
    assert res.errcode == out.errcode == 0
    assert res.evaluations == len(out.history)
    n = min(20, len(out.history))
    np.testing.assert_allclose(res.history[:n], out.history[:n], rtol=1e-8)
    assert float(np.max(np.abs(rho / ro - 1))) < 1e-8


@pytest.mark.parametrize("case", ["octane", "water_octane"])
def test_converge_interface_and_gamma(case):
    import cdft_b200 as cd
    sp, so = (S.octane_vle if case == "octane" else S.water_octane_lle)(N=256)
    rho = cd.initialize_profiles(sp)
    rho_o = so.initialize_profiles()
    # the seeds agree up to the two independent critical-temperature estimates
    np.testing.assert_allclose(rho, rho_o, rtol=1e-3)
    rho0 = rho.copy()
    kw = dict(beta=0.01, tol=1e-12, anderson_m=5, maxit=10000)   # converge! defaults except tol
    res = cd.converge(sp, rho, **kw)
    ro, out = so.converge(rho0, **kw)
    assert res.idid and out.idid, (res, out.errcode)
    err, shifts = _aligned_log_diff(rho, ro)
    assert err < 1e-9, (err, shifts)
    assert max(abs(x) for x in shifts) < 1e-3
    g = cd.surface_tension(sp, rho) / 2
    go = so.surface_tension(ro) / 2
    assert g == pytest.approx(go, rel=1e-9)
    assert g > 0


def test_errcodes_match_oracle():
    import cdft_b200 as cd
    from oracle import pcsaft_bulk as pb
    pm, om = S.models(["methane"])
    rb = pb.density(om, 1e7, 150.0, [1.0])
    L = om.length_scale()
    # uniform bulk profile is already the fixed point -> -1
    sysp = cd.DFTSystem(pm, cd.Uniform1DCart((1e7, 150.0), [rb], [-5 * L, 5 * L], 32))
    rho = cd.initialize_profiles(sysp)
    assert cd.converge(sysp, rho, beta=0.1, tol=1e-8).errcode == -1
    # maxit exhausted -> 10
    sp, so = S.methane_wall(N=101)
    rho = cd.initialize_profiles(sp)
    r0 = rho.copy()
    res = cd.converge(sp, rho, beta=0.1, tol=1e-14, anderson_m=5, maxit=7)
    _, out = so.converge(r0, beta=0.1, tol=1e-14, anderson_m=5, maxit=7)
    assert res.errcode == out.errcode == 10
    assert res.evaluations == len(out.history)
    # pure damped Picard (m = 0) on a dilute slit pore, where it converges
    sp, so = S.slit_pore(2e-9, 1e3, 100)
    rho = cd.initialize_profiles(sp)
    r0 = rho.copy()
    res = cd.converge(sp, rho, beta=0.1, tol=1e-8, anderson_m=0, maxit=2000)
    ro, out = so.converge(r0, beta=0.1, tol=1e-8, anderson_m=0, maxit=2000)
    assert res.errcode == out.errcode == 0
    assert abs(res.evaluations - len(out.history)) <= 2
    assert float(np.max(np.abs(rho / ro - 1))) < 1e-8


@pytest.mark.parametrize("engine", ["grid", "persistent"])
def test_batch_equals_individual_bitwise(engine):
    """Uneven slit pores converged in one batch give bit-identical results to
    converging each alone (deterministic reductions, per-system chunking)."""
    import cdft_b200 as cd
    cases = [(2e-9, 1e3, 100), (4e-9, 1e5, 180), (8e-9, 1e7, 400), (3e-9, 1e6, 137)]
    systems, rhos = [], []
    for H, p, N in cases:
        sp, _ = S.slit_pore(H, p, N)
        systems.append(sp)
        rhos.append(cd.initialize_profiles(sp))
    singles = []
    for sp, r in zip(systems, rhos):
        rr = r.copy()
        singles.append((rr, cd.converge(sp, rr, beta=0.1, tol=1e-10, anderson_m=5, engine=engine)))
    batch = [r.copy() for r in rhos]
    results = cd.batch_converge(systems, batch, beta=0.1, tol=1e-10, anderson_m=5, engine=engine)
    for (rr, rs), rb, res in zip(singles, batch, results):
        assert res.errcode == rs.errcode == 0
        assert res.evaluations == rs.evaluations
        assert np.array_equal(rr, rb)


def test_engines_agree():
    """Grid and persistent engines run the same aasol algorithm with different
    summation orders (the persistent engine's convolutions run on the FP64
    tensor cores).  Their residual histories agree over the first evaluations,
    until the Anderson steps amplify those rounding differences (within ~40
    evaluations on the 8 nm pore at 1e7 Pa), and both reach the same fixed point."""
    import cdft_b200 as cd
    for H, p, N in [(2e-9, 1e3, 100), (8e-9, 1e7, 400), (5e-9, 7.2e5, 300)]:
        sp, _ = S.slit_pore(H, p, N)
        r0 = cd.initialize_profiles(sp)
        a, b = r0.copy(), r0.copy()
        ra = cd.converge(sp, a, beta=0.1, tol=1e-10, anderson_m=5, engine="grid")
        rb = cd.converge(sp, b, beta=0.1, tol=1e-10, anderson_m=5, engine="persistent")
        assert ra.errcode == rb.errcode == 0
        k = min(12, ra.evaluations, rb.evaluations)
        np.testing.assert_allclose(ra.history[:k], rb.history[:k], rtol=1e-8, atol=1e-12 * ra.history[0])
        assert float(np.max(np.abs(a / b - 1))) < 1e-8


@pytest.mark.parametrize("engine", ["grid", "persistent"])
def test_mixed_precision_reaches_fp64_fixed_point(engine):
    """Mixed plans: FP32 convolutions/Phi until the residual fell by 1e-5, then an
    FP64 polish.  The result is the FP64 fixed point: profiles 1e-9, adsorption
    and the surface grand potential within 1e-9 of the FP64 path."""
    import cdft_b200 as cd
    for H, p, N in [(3e-9, 1e5, 160), (6e-9, 2.7e6, 310)]:
        s64, _ = S.slit_pore(H, p, N)
        s32, _ = S.slit_pore(H, p, N, precision="mixed")
        r0 = cd.initialize_profiles(s64)
        a, b = r0.copy(), r0.copy()
        ra = cd.converge(s64, a, beta=0.1, tol=1e-10, anderson_m=5, engine=engine)
        rb = cd.converge(s32, b, beta=0.1, tol=1e-10, anderson_m=5, engine=engine)
        assert ra.errcode == 0 and rb.errcode == 0
        assert float(np.max(np.abs(a / b - 1))) < 1e-8
        assert cd.adsorption(s32, b)[0] == pytest.approx(cd.adsorption(s64, a)[0], rel=1e-9)
        assert cd.surface_tension(s32, b) == pytest.approx(cd.surface_tension(s64, a), rel=1e-8)


def test_mixed_dfdrho_close_to_fp64():
    """FP32 convolutions and Phi: dF/drho within FP32 accuracy of the FP64 path."""
    import cdft_b200 as cd
    rng = np.random.default_rng(5)
    s64, so = S.water_octane_lle(N=256)
    s32 = cd.DFTSystem(s64.model, s64.structure, None, cd.DFTOptions("mixed"))
    rho = S.random_smooth_profile(s64, rng)
    d64 = cd.dFdrho_res(s64, rho)
    d32 = cd.dFdrho_res(s32, rho)
    for i in range(2):
        assert _rel(d32[i], d64[i]) < 2e-5, _rel(d32[i], d64[i])


@pytest.mark.parametrize("case", ["wall", "lle", "sphr", "3d"])
def test_device_integrals_match_host_quadrature(case):
    """cdft_batch_integrals (F_res, F_ideal, int rho, int 1 on the device, compensated sums)
    against the host Simpson / radial quadrature of the same profile and the oracle's
    surface_tension numerator and adsorption."""
    import cdft_b200 as cd
    rng = np.random.default_rng(11)
    so = None
    if case == "wall":
        sp, so = S.methane_wall(N=201)
        rho = cd.initialize_profiles(sp)
    elif case == "lle":
        sp, so = S.water_octane_lle(N=256)
        rho = S.random_smooth_profile(sp, rng)
    elif case == "sphr":
        from oracle import pcsaft_bulk as pb
        pm, om = S.models(["methane"])
        rb = pb.density(om, 1e7, 150.0, [1.0])
        sp = cd.DFTSystem(pm, cd.Uniform1DSphr((1e7, 150.0), [rb], [0.0, 10 * om.sigma[0]], 121),
                          cd.HardCore(1.5 * om.sigma[0]))
        rho = cd.initialize_profiles(sp)
    else:
        from oracle import pcsaft_bulk as pb
        pm, om = S.models(["argon"])
        rb = 0.021e30 / pb.N_A
        box = 8.0 * om.sigma[0]
        sp = cd.DFTSystem(pm, cd.Uniform3DCart((1e5, 100.0), [rb], [0.0, box], 32), None)
        x = np.arange(32) / 32
        rho = cd.initialize_profiles(sp) * (1 + 0.1 * np.sin(2 * np.pi * x))[None, None, None, :]
        rho = np.ascontiguousarray(rho)
    q = cd.batch_integrals([sp], [rho])[0]
    st = sp.structure
    T = st.conditions[1]
    fid = (cd.N_A * rho * (np.log(rho) - 1.5 * np.log(T) - 1)).sum(axis=0)
    assert q["F_ideal"] == pytest.approx(cd.integrate(fid, st), rel=1e-12)
    for i in range(sp.nc):
        assert q["int_rho"][i] == pytest.approx(cd.integrate(rho[i], st), rel=1e-12)
    assert q["int_one"] == pytest.approx(cd.integrate(np.ones(st.grid_shape), st), rel=1e-12)
    assert q["F_res"] == pytest.approx(cd.F_res(sp, rho), rel=1e-12)
    if so is not None:
        assert cd.surface_tension(sp, rho) == pytest.approx(so.surface_tension(rho), rel=1e-10)
        assert cd.adsorption(sp, rho) == pytest.approx(so.adsorption(rho), rel=1e-12)


def test_persistent_anderson_warp_and_block_paths_agree():
    """The persistent engine's Anderson section on one warp (systems up to
    pers_warp_aa_max_elem elements) and on the whole block reduce in different orders:
    both reach the oracle's fixed point."""
    import cdft_b200 as cd
    sp, so = S.methane_wall(N=201)
    ro, out = so.converge(cd.initialize_profiles(sp), beta=0.1, tol=1e-13, anderson_m=5)
    old = cd.tuning("pers_warp_aa_max_elem")
    try:
        for thr in (0, 1 << 20):
            cd.tuning("pers_warp_aa_max_elem", thr)
            rho = cd.initialize_profiles(sp)
            res = cd.converge(sp, rho, beta=0.1, tol=1e-13, anderson_m=5, engine="persistent")
            assert res.errcode == 0
            assert float(np.max(np.abs(rho / ro - 1))) < 1e-9, thr
    finally:
        cd.tuning("pers_warp_aa_max_elem", old)


def test_persistent_cluster_pairs_equal_single_ctas_bitwise():
    """Two CTAs per system (a cluster of two splitting the convolution tasks and the Phi
    points) compute every value with the same code as one CTA per system: the 64-point
    isotherm converges to the same bits, with the same evaluation counts."""
    import bench
    import cdft_b200 as cd
    specs = bench.isotherm_specs(0)[::4]
    systems, rho0 = bench.build_systems(specs, "fp64")
    method = cd.AASol.for_system(None, **bench.SOLVER)
    old = cd.tuning("pers_cluster")
    out = {}
    try:
        for c in (0, 1):
            cd.tuning("pers_cluster", c)
            rr = [r.copy() for r in rho0]
            res = cd.batch_converge(systems, rr, method=method, engine="persistent")
            out[c] = (rr, [r.evaluations for r in res], [r.errcode for r in res])
    finally:
        cd.tuning("pers_cluster", old)
    assert out[0][1] == out[1][1] and out[0][2] == out[1][2]
    for a, b in zip(out[0][0], out[1][0]):
        assert np.array_equal(a, b)
