"""The envelope theorem behind cdft_grad_params, on the oracle (CPU).

At a converged profile the grand potential is stationary in rho, so its parameter
derivative is k_B T dF_res/dtheta|rho + R T int rho dV/dtheta - dmu/dtheta int rho +
dp/dtheta int 1, with no derivative of the profile.  That holds for the discrete functional
whose gradient the pointwise Euler-Lagrange equation is: every integral summed with uniform
weights dz (the adjoint of the periodic convolution).  Methane in a graphite slit, where the
adsorbed layers are sharp on the grid: with uniform weights the formula equals central
differences through converge; with the Simpson weights of surface_tension it does not."""
import numpy as np

import _systems as S
from oracle import functional as fn, pcsaft_bulk as pb

T, H, N = 150.0, 3e-9, 150
KW = dict(beta=0.1, tol=1e-12, anderson_m=5)


def _setup():
    pm, _ = S.models(["methane"])
    rb = pm.stable_density(1e5, T, [1.0])
    s = pm.sigma[0]
    P = S.PARAMS["methane"]
    return rb, (0.7 * s, H - 0.7 * s), np.array([P["sigma"], P["eps"], P["m"]])


def _build(th, rb, bounds):
    m = pb.PCSAFTModel(["methane"], [th[2]], [th[0]], [th[1]])
    p = pb.pressure(m, [rb], T)
    return fn.DFTSystem(m, fn.Structure((p, T), [rb], [bounds], (N,)), [fn.SteeleWall.graphite(H)]), m, p


def _mu(m, rb):
    return pb.R_GAS * T * (np.log(rb) - 1.5 * np.log(T) + pb.mu_res(m, [rb], T)[0])


def _omega(so, m, p, rho, rb, quad):
    F = quad(so.phi(so.weighted_densities(rho))) / so.L ** 3 + \
        quad(pb.N_A * rho[0] * (np.log(rho[0]) - 1.5 * np.log(T) - 1))
    return (F * pb.K_B * T - _mu(m, rb) * quad(rho[0]) + p * quad(np.ones(N))
            + pb.N_A * pb.K_B * T * quad(rho[0] * so.vext[0]))


def test_envelope_formula_is_exact_with_uniform_weights():
    rb, bounds, theta0 = _setup()
    so, m0, p0 = _build(theta0, rb, bounds)
    with np.errstate(all="ignore"):
        rho, out = so.converge(so.initialize_profiles(), **KW)
    assert out.errcode == 0
    dz = (bounds[1] - bounds[0]) / N
    uniform = lambda f: dz * np.sum(f)   # noqa: E731
    fd = {"uniform": np.zeros(3), "simpson": np.zeros(3)}
    env = {"uniform": np.zeros(3), "simpson": np.zeros(3)}
    for name, quad in (("uniform", uniform), ("simpson", so.integral)):
        for t in range(3):
            h = 1e-6 * theta0[t]
            vals, Fs, Vs, mus, ps = [], [], [], [], []
            for sg in (1.0, -1.0):
                th = theta0.copy()
                th[t] += sg * h
                so2, m2, p2 = _build(th, rb, bounds)
                with np.errstate(all="ignore"):
                    r2, _ = so2.converge(rho.copy(), **KW)
                vals.append(_omega(so2, m2, p2, r2, rb, quad))
                Fs.append(quad(so2.phi(so2.weighted_densities(rho))) / so2.L ** 3)
                Vs.append(quad(rho[0] * so2.vext[0]))
                mus.append(_mu(m2, rb))
                ps.append(p2)
            d = lambda v: (v[0] - v[1]) / (2 * h)   # noqa: E731
            fd[name][t] = d(vals)
            env[name][t] = (pb.K_B * T * d(Fs) + pb.N_A * pb.K_B * T * d(Vs) - d(mus) * quad(rho[0])
                            + d(ps) * quad(np.ones(N)))
    scale = np.max(np.abs(fd["uniform"]))
    assert np.max(np.abs(env["uniform"] - fd["uniform"])) < 1e-6 * scale
    # the Simpson-weighted grand potential is not stationary at the discrete fixed point
    assert np.max(np.abs(env["simpson"] - fd["simpson"])) > 1e-2 * np.max(np.abs(fd["simpson"]))
