"""Matched system builders: the same inputs for the CUDA path (cdft_b200) and
the CPU oracle, for the configurations the parity tests use.

Parameters are the explicit PC-SAFT sets of the benchmark configurations
(methane, n-octane, water 2B, argon); the Steele wall is graphite from the
reference's Steele database row.
"""
import functools

import numpy as np

from oracle import functional as fn
from oracle import pcsaft_bulk as pb

PARAMS = {
    "methane": dict(m=1.0, sigma=3.7039, eps=150.03),
    "octane": dict(m=3.8176, sigma=3.8373, eps=242.78),
    "water": dict(m=1.0656, sigma=3.0007, eps=366.51, assoc=(2500.7, 0.034868)),
    "argon": dict(m=1.0, sigma=3.4, eps=120.0),
    "ethanol": dict(m=2.3827, sigma=3.1771, eps=198.24, assoc=(2653.4, 0.032384)),
}


def cross_assoc(P):
    """Cross-association between every two self-associating components by the Elliott
    rule: eps_ij = (eps_i + eps_j)/2, kappa_ij sigma_ij^3 = sqrt(kappa_i sigma_i^3 kappa_j sigma_j^3)."""
    out = {}
    for i, a in enumerate(P):
        for j, b in enumerate(P):
            if j > i and "assoc" in a and "assoc" in b:
                sij = 0.5 * (a["sigma"] + b["sigma"])
                k = np.sqrt(a["assoc"][1] * b["assoc"][1]) * (np.sqrt(a["sigma"] * b["sigma"]) / sij) ** 3
                out[(i, j)] = (0.5 * (a["assoc"][0] + b["assoc"][0]), float(k))
    return out


def models(names):
    """(package PCSAFT, oracle PCSAFTModel) for the named components."""
    import cdft_b200 as cd
    P = [PARAMS[n] for n in names]
    m = [p["m"] for p in P]
    s = [p["sigma"] for p in P]
    e = [p["eps"] for p in P]
    assoc_pkg = {i: p["assoc"] for i, p in enumerate(P) if "assoc" in p}
    assoc_or = [(i, i, p["assoc"][0], p["assoc"][1]) for i, p in enumerate(P) if "assoc" in p]
    cross = cross_assoc(P)
    assoc_or += [(i, j, e_, k_) for (i, j), (e_, k_) in cross.items()]
    om = pb.PCSAFTModel(names, m, s, e, assoc=assoc_or)
    if cross:
        return cd.PCSAFT(names, m, s, e, assoc=assoc_pkg, assoc_cross=cross), om
    return cd.PCSAFT(names, m, s, e, assoc=assoc_pkg), om


def pair(names, conditions, rho_bulk, bounds, N, kind="uniform", rho_bulk2=None, walls=(), precision="fp64"):
    """Build (package system, oracle system)."""
    import cdft_b200 as cd
    pm, om = models(names)
    if kind == "uniform":
        st = cd.Uniform1DCart(conditions, rho_bulk, bounds, N)
    else:
        st = cd.TwoPhase1DCart(conditions, rho_bulk, rho_bulk2, bounds, N)
    fields = [cd.Steele(["graphite"], w) for w in walls]
    sysp = cd.DFTSystem(pm, st, fields or None, cd.DFTOptions(precision))
    ost = fn.Structure(conditions, rho_bulk, [tuple(bounds)], (N,), kind=kind, rho_bulk2=rho_bulk2)
    syso = fn.DFTSystem(om, ost, [fn.SteeleWall.graphite(w) for w in walls])
    return sysp, syso


def methane_wall(N=201, width=0.0, precision="fp64", p=1e7, T=150.0):
    """Methane liquid at 150 K, 10 MPa next to a graphite Steele wall on [0.5 sigma, 4.5 sigma]."""
    _, om = models(["methane"])
    rb = pb.density(om, p, T, [1.0])
    s = om.sigma[0]
    return pair(["methane"], (p, T), [rb], (0.5 * s, 4.5 * s), N, walls=(width,), precision=precision)


def slit_pore(H, p, N, T=150.0, precision="fp64"):
    """Methane in a graphite slit of width H (m): bounds [0.7 sigma, H - 0.7 sigma]
    as adsorption(model, surface, p, T) builds them (adsorption.jl:48-65)."""
    _, om = models(["methane"])
    try:
        rb = pb.density(om, p, T, [1.0], "vapour")
    except RuntimeError:
        rb = pb.density(om, p, T, [1.0], "liquid")
    s = om.sigma[0]
    return pair(["methane"], (p, T), [rb], (0.7 * s, H - 0.7 * s), N, walls=(H,), precision=precision)


@functools.lru_cache(maxsize=None)
def _vle(name, T):
    _, om = models([name])
    return pb.saturation_pure(om, T)


@functools.lru_cache(maxsize=None)
def _lle(names, p, T):
    _, om = models(list(names))
    x1, x2 = pb.lle_binary(om, p, T)
    return tuple(pb.density(om, p, T, x1) * x1), tuple(pb.density(om, p, T, x2) * x2)


def octane_vle(N=256, box_sigmas=40.0, T=298.15):
    _, om = models(["octane"])
    psat, rl, rv = _vle("octane", T)
    s = om.sigma[0]
    half = box_sigmas * s / 2
    return pair(["octane"], (psat, T), [rl], (-half, half), N, kind="twophase", rho_bulk2=[rv])


def water_octane_lle(N=256, box_sigmas=60.0, T=298.15, p=1e5):
    _, om = models(["water", "octane"])
    r1, r2 = _lle(("water", "octane"), p, T)
    s = om.sigma[0]
    half = box_sigmas * s / 2
    return pair(["water", "octane"], (p, T), list(r1), (-half, half), N, kind="twophase", rho_bulk2=list(r2))


def water_ethanol_wall(N=150, x=(0.5, 0.5), p=1e5, T=298.15, width=0.0, precision="fp64"):
    """Liquid water + ethanol (self- and cross-association: 4 site pairs, the general
    association path, as the reference's test/test_models.jl:171-188 case) next to a
    graphite Steele wall on [0.5 sigma_w, 4.5 sigma_w]."""
    _, om = models(["water", "ethanol"])
    x = np.asarray(x, dtype=float)
    rb = x * pb.density(om, p, T, x, "liquid")
    s = om.sigma[0]
    return pair(["water", "ethanol"], (p, T), list(rb), (0.5 * s, 4.5 * s), N, walls=(width,), precision=precision)


def random_smooth_profile(sysp, rng, amp=0.3):
    """A positive, smooth non-uniform profile around the bulk densities."""
    st = sysp.structure
    N = st.ngrid[0]
    x = np.linspace(0, 1, N)
    out = np.empty((sysp.nc, N))
    for i in range(sysp.nc):
        ph = rng.random(3) * 2 * np.pi
        out[i] = st.rho_bulk[i] * (1 + amp * (np.sin(2 * np.pi * x + ph[0]) + 0.5 * np.sin(6 * np.pi * x + ph[1])
                                            + 0.25 * np.cos(14 * np.pi * x + ph[2])))
    return out


def aligned_log_diff(rho, ref):
    """Max |ln rho - ln ref| after removing the interface displacements.

    A periodic box holding two interfaces at coexistence has two (near-)zero
    modes: a common translation and a breathing mode (one phase grows while
    the other shrinks), so two correct solvers can stop with the interfaces a
    tiny distance apart.  Each half of the box holds one interface (the seed
    puts them at +-H/4 around the centre); one displacement per half is fitted
    by least squares with the exact spectral derivative of the periodic
    N-point problem and removed before comparing.  Returns (max diff, shifts
    in grid units)."""
    N = ref.shape[-1]
    k = np.fft.fftfreq(N) * N
    lr = np.log(ref)
    D = np.real(np.fft.ifft(2j * np.pi * k / N * np.fft.fft(lr, axis=-1), axis=-1))
    d = np.log(rho) - lr
    r = d.copy()
    shifts = []
    for half in (slice(0, N // 2), slice(N // 2, N)):
        Dh, dh = D[:, half], d[:, half]
        sh = -np.sum(dh * Dh) / np.sum(Dh * Dh)
        r[:, half] = dh + sh * Dh
        shifts.append(float(sh))
    return float(np.max(np.abs(r))), shifts
