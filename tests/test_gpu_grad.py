"""Parameter gradients through the C ABI, against central finite differences.

theta = (sigma_k [A], eps_k/k_B [K], m_k) for every component k.  The reference has
no parameter gradient (it differentiates f_res in the weighted densities only,
models.jl:355-411), so the checks are central differences:

- dF_res/dtheta at a fixed profile against the oracle's F_res with perturbed
  parameters (FMT, chain, dispersion, association, and the kernels through the
  hard-sphere diameter);
- d gamma/dtheta of the water/n-octane liquid-liquid interface (the differentiation
  configuration, on a shorter grid) against gamma recomputed through the whole
  pipeline at theta +- h: bulk coexistence, converge from the converged profile,
  surface tension.
"""
import numpy as np
import pytest

import _systems as S

pytestmark = pytest.mark.gpu


def _oracle_model(names, theta):
    from oracle import pcsaft_bulk as pb
    t = np.asarray(theta, dtype=float).reshape(-1, 3)
    P = [S.PARAMS[n] for n in names]
    assoc = [(i, i, p["assoc"][0], p["assoc"][1]) for i, p in enumerate(P) if "assoc" in p]
    return pb.PCSAFTModel(names, t[:, 2], t[:, 0], t[:, 1], assoc=assoc)


CASES = {
    "methane_wall": (["methane"], lambda: S.methane_wall(N=201)),
    "octane_vle": (["octane"], lambda: S.octane_vle(N=256)),
    "water_octane_lle": (["water", "octane"], lambda: S.water_octane_lle(N=256)),
}


@pytest.mark.parametrize("case", list(CASES))
def test_F_res_grad_matches_oracle_fd(case):
    """Hand-written parameter gradient of F_res vs the oracle's central differences
    (relative step 1e-5: truncation ~1e-10, rounding ~1e-11 relative)."""
    import cdft_b200 as cd
    from oracle import functional as fn
    names, build = CASES[case]
    sp, so = build()
    rng = np.random.default_rng(5)
    rho = S.random_smooth_profile(sp, rng, amp=0.2)
    g = cd.F_res_grad(sp, rho).ravel()
    theta0 = sp.model.theta()
    fd = np.empty_like(theta0)
    for t in range(theta0.size):
        h = 1e-5 * abs(theta0[t])
        vals = []
        for sgn in (1.0, -1.0):
            th = theta0.copy()
            th[t] += sgn * h
            st = fn.DFTSystem(_oracle_model(names, th), so.structure, so.walls)
            vals.append(st.F_res(rho))
        fd[t] = (vals[0] - vals[1]) / (2 * h)
    # each entry against its own size, floored at 1e-4 of the largest: the differences
    # carry rounding noise eps |F_res| / h, which for the smallest entries (a component's
    # sigma in a mixture dominated by the other) is ~1e-6 of the entry itself
    scale = np.maximum(np.abs(fd), 1e-4 * np.max(np.abs(fd)))
    err = np.abs(g - fd) / scale
    assert float(np.max(err)) < 1e-6, (g, fd)


def test_grad_params_scope():
    """Planar Steele walls are differentiated (their dV/dtheta enters the gradient); radial
    grids have no parameter gradient and are refused."""
    import cdft_b200 as cd
    from cdft_b200._lib import CDFTError
    sp, _ = S.methane_wall(N=101)
    rho = cd.initialize_profiles(sp)
    cd.F_res_grad(sp, rho)   # F_res itself carries no external field
    g = cd.grad_params(sp, rho)
    assert g.shape == (1, 3) and np.all(np.isfinite(g))
    pm, _ = S.models(["argon"])
    r1 = cd.DFTSystem(pm, cd.Uniform1DSphr((1e5, 100.0), [0.021e30 / cd.N_A], [0.0, 8 * 3.4e-10], 64))
    with pytest.raises(CDFTError):
        cd.F_res_grad(r1, cd.initialize_profiles(r1))
    r1.close()


def _lle_system(model, N, box_sigmas=60.0, T=298.15, p=1e5):
    import cdft_b200 as cd
    x1, x2 = model.lle(p, T)
    r1 = model.molar_density(p, T, x1, "liquid") * x1
    r2 = model.molar_density(p, T, x2, "liquid") * x2
    s = model.sigma[0]
    half = box_sigmas * s / 2
    st = cd.TwoPhase1DCart((p, T), list(r1), list(r2), [-half, half], N)
    return cd.DFTSystem(model, st)


@pytest.mark.parametrize("N", [256, 4096])
def test_dgamma_dtheta_water_octane_matches_fd(N):
    """d gamma/dtheta (adjoint at the converged profile + coexistence sensitivity) vs
    central differences of gamma through bulk LLE, converge and surface tension; 4096
    points over 60 sigma is the differentiation configuration itself.  The difference step
    is 1e-5 relative: with converge's 1e-12 tolerance (about 1e-10 relative in gamma) a 1e-6
    step would leave ~5e-5 of noise in the quotient."""
    import cdft_b200 as cd
    pm, _ = S.models(["water", "octane"])
    kw = dict(beta=0.01, tol=1e-12, anderson_m=5, maxit=20000)
    sys0 = _lle_system(pm, N)
    rho0 = cd.initialize_profiles(sys0)
    res = cd.converge(sys0, rho0, **kw)
    assert res.errcode == 0
    grad = cd.dgamma_dtheta(sys0, rho0).ravel()
    theta0 = pm.theta()
    fd = np.empty_like(theta0)
    for t in range(theta0.size):
        h = 1e-5 * abs(theta0[t])
        vals = []
        for sgn in (1.0, -1.0):
            th = theta0.copy()
            th[t] += sgn * h
            mdl = pm.with_theta(th)
            st = _lle_system(mdl, N)
            r = rho0.copy()
            rr = cd.converge(st, r, **kw)
            assert rr.errcode in (0, -1)
            vals.append(cd.surface_tension(st, r) / 2)
            st.close()
        fd[t] = (vals[0] - vals[1]) / (2 * h)
    err = np.abs(grad - fd) / np.max(np.abs(fd))
    assert float(np.max(err)) < 1e-5, (grad, fd)


def test_dgrand_potential_dtheta_slit_pore_matches_fd():
    """Methane in a graphite slit (two Steele walls): d Omega/d theta of the grand potential
    including the wall energy, with the walls' own dependence on sigma_i and eps_i, against
    central differences (step 1e-6 relative) through converge at fixed bulk density (mu and
    p follow the parameters).  Omega in the uniform quadrature, the discrete functional the
    converged profile is stationary in: the adsorbed layers are sharp on this grid, and
    surface_tension's Simpson weights would add a discretisation term the envelope theorem
    does not see (the oracle shows the same, and agreement to all digits with uniform weights)."""
    import cdft_b200 as cd
    pm, _ = S.models(["methane"])
    T, H, p0, N = 150.0, 3e-9, 1e5, 150
    rb = pm.stable_density(p0, T, [1.0])
    s = pm.sigma[0]
    bounds = [0.7 * s, H - 0.7 * s]
    kw = dict(beta=0.1, tol=1e-12, anderson_m=5, maxit=20000)

    def build(model):
        st = cd.Uniform1DCart((model.pressure([rb], T), T), [rb], bounds, N)
        return cd.DFTSystem(model, st, cd.Steele(["graphite"], H))

    sys0 = build(pm)
    rho0 = cd.initialize_profiles(sys0)
    assert cd.converge(sys0, rho0, **kw).errcode == 0
    theta0 = pm.theta()
    dmu = np.zeros((1, 3))
    dp = np.zeros(3)
    fd = np.zeros(3)
    for t in range(3):
        h = 1e-6 * abs(theta0[t])
        vals, mus, ps = [], [], []
        for sgn in (1.0, -1.0):
            th = theta0.copy()
            th[t] += sgn * h
            mdl = pm.with_theta(th)
            mus.append(mdl.chemical_potential([rb], T)[0])
            ps.append(mdl.pressure([rb], T))
            st = build(mdl)
            r = rho0.copy()
            assert cd.converge(st, r, **kw).errcode in (0, -1)
            vals.append(cd.grand_potential(st, r, quadrature="uniform"))
            st.close()
        fd[t] = (vals[0] - vals[1]) / (2 * h)
        dmu[0, t] = (mus[0] - mus[1]) / (2 * h)
        dp[t] = (ps[0] - ps[1]) / (2 * h)
    grad = cd.grad_params(sys0, rho0, dmu, dp).ravel()
    err = np.abs(grad - fd) / np.max(np.abs(fd))
    assert float(np.max(err)) < 1e-5, (grad, fd)


def _argon_box(N=32, box_sigmas=8.0, solutes=False):
    import cdft_b200 as cd
    from oracle import functional as fn
    pm, om = S.models(["argon"])
    s = om.sigma[0]
    box = box_sigmas * s
    rb = 0.021e30 / cd.N_A
    field = None
    if solutes:
        centres = cd.HardSphereSolutes.seeded(4, 1.2 * s, box, 2 * box / N, seed=1)
        field = cd.HardSphereSolutes(centres, 1.2 * s)
    sp = cd.DFTSystem(pm, cd.Uniform3DCart((1e5, 100.0), [rb], [0.0, box], N), field)
    st = fn.Structure((1e5, 100.0), [rb], [(0.0, box)] * 3, (N, N, N))
    return sp, st, pm, rb, box


def test_F_res_grad_3d_matches_oracle_fd():
    """The 3D parameter gradient of F_res (explicit terms and the kernels' dependence on the
    diameter through the FFT pipeline with derivative tables) against the oracle's central
    differences of its 3D F_res, argon on a 32^3 box with a smooth non-uniform profile."""
    import cdft_b200 as cd
    from oracle import functional as fn
    sp, st, pm, rb, box = _argon_box()
    N = 32
    x = np.arange(N) / N
    Z, Y, X = np.meshgrid(x, x, x, indexing="ij")
    rho = rb * (1 + 0.2 * np.sin(2 * np.pi * X) * np.cos(2 * np.pi * Y) + 0.1 * np.sin(4 * np.pi * Z))[None]
    rho = np.ascontiguousarray(rho)
    g = cd.F_res_grad(sp, rho).ravel()
    theta0 = pm.theta()
    fd = np.empty_like(theta0)
    for t in range(theta0.size):
        h = 1e-5 * abs(theta0[t])
        vals = []
        for sgn in (1.0, -1.0):
            th = theta0.copy()
            th[t] += sgn * h
            vals.append(fn.DFTSystem(_oracle_model(["argon"], th), st).F_res(rho))
        fd[t] = (vals[0] - vals[1]) / (2 * h)
    scale = np.maximum(np.abs(fd), 1e-4 * np.max(np.abs(fd)))
    assert float(np.max(np.abs(g - fd) / scale)) < 1e-6, (g, fd)
    sp.close()


def test_dgrand_potential_dtheta_3d_solutes_matches_fd():
    """d Omega / d theta of a converged 32^3 argon box with hard solutes (the uniform-weight
    grand potential the converged profile is stationary in) against central differences
    through converge at fixed bulk density."""
    import cdft_b200 as cd
    sp, st, pm, rb, box = _argon_box(solutes=True)
    T = 100.0
    kw = dict(beta=0.1, tol=1e-11, anderson_m=10, maxit=2000)

    def build(model):
        cen = sp.external_field[0].centres
        return cd.DFTSystem(model, cd.Uniform3DCart((model.pressure([rb], T), T), [rb], [0.0, box], 32),
                            cd.HardSphereSolutes(cen, sp.external_field[0].radius))

    sys0 = build(pm)
    rho0 = cd.initialize_profiles(sys0)
    assert cd.converge(sys0, rho0, **kw).errcode == 0
    theta0 = pm.theta()
    dmu, dp, fd = np.zeros((1, 3)), np.zeros(3), np.zeros(3)
    for t in range(3):
        h = 1e-6 * abs(theta0[t])
        vals, mus, ps = [], [], []
        for sgn in (1.0, -1.0):
            th = theta0.copy()
            th[t] += sgn * h
            mdl = pm.with_theta(th)
            mus.append(mdl.chemical_potential([rb], T)[0])
            ps.append(mdl.pressure([rb], T))
            s2 = build(mdl)
            r = rho0.copy()
            assert cd.converge(s2, r, **kw).errcode in (0, -1)
            vals.append(cd.grand_potential(s2, r, quadrature="uniform"))
            s2.close()
        fd[t] = (vals[0] - vals[1]) / (2 * h)
        dmu[0, t] = (mus[0] - mus[1]) / (2 * h)
        dp[t] = (ps[0] - ps[1]) / (2 * h)
    grad = cd.grad_params(sys0, rho0, dmu, dp).ravel()
    err = np.abs(grad - fd) / np.max(np.abs(fd))
    assert float(np.max(err)) < 1e-5, (grad, fd)
    sys0.close()
    sp.close()
