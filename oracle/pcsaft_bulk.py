"""Independent bulk PC-SAFT (TEST ORACLE), written from the published equations.

Gross & Sadowski, Ind. Eng. Chem. Res. 40 (2001) 1244 (hard chain + dispersion)
and Ind. Eng. Chem. Res. 41 (2002) 5510 (association), with the
Boublik--Mansoori hard-sphere term.  It replaces the Clapeyron.jl calls the
reference makes on the converge! path (src/models/DFT/SAFT/PCSAFT/PCSAFT.jl:65-72
``get_species``: the hard-sphere diameter ``d`` and ``VT_chemical_potential_res``)
and in the property methods (``volume``, ``bubble_pressure``, ``tp_flash``,
``crit_pure``; src/methods/*.jl, src/structure/two_phase.jl:1-6).

Everything here is deliberately NOT derived from the DFT functional: the
bulk-consistency tests compare the functional's dF/drho at a uniform profile
with ``mu_res`` computed here.

Units: densities in mol/m^3, lengths in m, energies in K (eps/k_B), T in K.
Derivatives use the complex-step method (all functions accept complex input).
"""
import numpy as np

N_A = 6.02214076e23
K_B = 1.380649e-23
R_GAS = N_A * K_B

# Universal constants of the PC-SAFT dispersion integrals, Gross & Sadowski
# (2001) Table 1: rows i = 0..6, columns (a0i, a1i, a2i) / (b0i, b1i, b2i).
# The reference carries the same published table (PCSAFT.jl:86-103).
PCSAFT_A = np.array([
    [0.9105631445, -0.3084016918, -0.0906148351],
    [0.6361281449, 0.1860531159, 0.4527842806],
    [2.6861347891, -2.5030047259, 0.5962700728],
    [-26.547362491, 21.419793629, -1.7241829131],
    [97.759208784, -65.25588533, -4.1302112531],
    [-159.59154087, 83.318680481, 13.77663187],
    [91.297774084, -33.74692293, -8.6728470368],
])
PCSAFT_B = np.array([
    [0.7240946941, -0.5755498075, 0.0976883116],
    [2.2382791861, 0.6995095521, -0.2557574982],
    [-4.0025849485, 3.892567339, -9.155856153],
    [-21.003576815, -17.215471648, 20.642075974],
    [26.855641363, 192.67226447, -38.804430052],
    [206.55133841, -161.82646165, 93.626774077],
    [-355.60235612, -165.20769346, -29.666905585],
])


class PCSAFTModel:
    """Pure-component PC-SAFT parameters plus binary interaction and 2B association.

    ``assoc`` is a list of (i, j, eps_AB [K], kappa_AB) self-association pairs
    between site A of component i and site B of component j (one A and one B
    site per associating molecule: the 2B scheme).
    """

    def __init__(self, names, m, sigma_A, eps_K, kij=None, assoc=None):
        self.names = list(names)
        self.m = np.asarray(m, dtype=np.float64)
        self.sigma = np.asarray(sigma_A, dtype=np.float64) * 1e-10
        self.eps = np.asarray(eps_K, dtype=np.float64)
        nc = len(self.m)
        self.kij = np.zeros((nc, nc)) if kij is None else np.asarray(kij, dtype=np.float64)
        self.assoc = list(assoc or [])
        self.sigma_ij = 0.5 * (self.sigma[:, None] + self.sigma[None, :])
        self.eps_ij = np.sqrt(self.eps[:, None] * self.eps[None, :]) * (1.0 - self.kij)

    @property
    def nc(self):
        return len(self.m)

    def split_pure(self, i):
        assoc = [(0, 0, e, k) for (a, b, e, k) in self.assoc if a == i and b == i]
        return PCSAFTModel([self.names[i]], [self.m[i]], [self.sigma[i] * 1e10], [self.eps[i]], assoc=assoc)

    def length_scale(self):
        # length_scale(model::SAFTModel) = maximum(sigma), src/models/DFT/SAFT/PCSAFT/PCSAFT.jl:79-81
        return float(np.max(self.sigma_ij))

    def hs_diameter(self, T):
        # Gross & Sadowski (2001) eq. 3; Clapeyron's d(model, V, T, z)
        return self.sigma * (1.0 - 0.12 * np.exp(-3.0 * self.eps / T))


def _assoc_X(model, rho_n, T, d, zeta2, zeta3):
    """Fractions of non-bonded sites for the 2B pairs (complex-step safe)."""
    nc = model.nc
    # sites: index 2*i (A) and 2*i+1 (B) of component i; only listed pairs bond
    ns = 2 * nc
    cplx = np.iscomplexobj(rho_n) or np.iscomplexobj(zeta3)
    delta = np.zeros((ns, ns), dtype=complex if cplx else float)
    for (i, j, eAB, kAB) in model.assoc:
        dij = d[i] * d[j] / (d[i] + d[j])
        g = 1.0 / (1.0 - zeta3) + dij * 3.0 * zeta2 / (1.0 - zeta3) ** 2 + dij ** 2 * 2.0 * zeta2 ** 2 / (1.0 - zeta3) ** 3
        D = model.sigma_ij[i, j] ** 3 * g * kAB * (np.exp(eAB / T) - 1.0)
        delta[2 * i, 2 * j + 1] = D
        delta[2 * j + 1, 2 * i] = D
        if i != j:
            delta[2 * j, 2 * i + 1] = D
            delta[2 * i + 1, 2 * j] = D
    rho_site = np.repeat(rho_n, 2)
    if all(i == j for (i, j, _, _) in model.assoc):
        # only 2B self-association: X_A = X_B = 2 / (1 + sqrt(1 + 4 rho_i Delta_i)) in closed form
        X = np.ones(ns, dtype=delta.dtype)
        for (i, _, _, _) in model.assoc:
            q = rho_n[i] * delta[2 * i, 2 * i + 1]
            X[2 * i] = X[2 * i + 1] = 2.0 / (1.0 + np.sqrt(1.0 + 4.0 * q))
        return X
    X = np.ones(ns, dtype=delta.dtype)
    for _ in range(5):  # a few damped substitutions, then Newton (quadratic)
        X = 0.5 * (X + 1.0 / (1.0 + delta @ (rho_site * X)))
    for _ in range(12):
        F = X * (1.0 + delta @ (rho_site * X)) - 1.0
        J = np.diag(1.0 + delta @ (rho_site * X)) + X[:, None] * delta * rho_site[None, :]
        X = X - np.linalg.solve(J, F)
    return X


def helmholtz_res_density(model, rho, T):
    """A_res / (V k_B T) in 1/m^3 at molar densities ``rho`` (mol/m^3)."""
    rho = np.asarray(rho)
    rho_n = rho * N_A
    rho_tot = np.sum(rho_n)
    x = rho_n / rho_tot
    m = model.m
    d = model.hs_diameter(T)
    zeta = [np.pi / 6.0 * np.sum(rho_n * m * d ** k) for k in range(4)]
    z0, z1, z2, z3 = zeta
    one_z3 = 1.0 - z3
    a_hs = (3.0 * z1 * z2 / one_z3 + z2 ** 3 / (z3 * one_z3 ** 2) + (z2 ** 3 / z3 ** 2 - z0) * np.log(one_z3)) / z0
    g_ii = 1.0 / one_z3 + (d / 2.0) * 3.0 * z2 / one_z3 ** 2 + (d / 2.0) ** 2 * 2.0 * z2 ** 2 / one_z3 ** 3
    mbar = np.sum(x * m)
    a_hc = mbar * a_hs - np.sum(x * (m - 1.0) * np.log(g_ii))
    eta = z3
    c1 = (mbar - 1.0) / mbar
    c2 = c1 * (mbar - 2.0) / mbar
    a_i = PCSAFT_A[:, 0] + c1 * PCSAFT_A[:, 1] + c2 * PCSAFT_A[:, 2]
    b_i = PCSAFT_B[:, 0] + c1 * PCSAFT_B[:, 1] + c2 * PCSAFT_B[:, 2]
    powers = np.array([eta ** i for i in range(7)])
    I1 = np.sum(a_i * powers)
    I2 = np.sum(b_i * powers)
    C1 = 1.0 / (1.0 + mbar * (8.0 * eta - 2.0 * eta ** 2) / (1.0 - eta) ** 4
                + (1.0 - mbar) * (20.0 * eta - 27.0 * eta ** 2 + 12.0 * eta ** 3 - 2.0 * eta ** 4)
                / ((1.0 - eta) * (2.0 - eta)) ** 2)
    mm = x[:, None] * x[None, :] * m[:, None] * m[None, :] * model.sigma_ij ** 3
    m2es3 = np.sum(mm * model.eps_ij / T)
    m2e2s3 = np.sum(mm * (model.eps_ij / T) ** 2)
    a_disp = -2.0 * np.pi * rho_tot * I1 * m2es3 - np.pi * rho_tot * mbar * C1 * I2 * m2e2s3
    a_assoc = 0.0
    if model.assoc:
        X = _assoc_X(model, rho_n, T, d, z2, z3)
        lnX = np.log(X) - X / 2.0 + 0.5
        for i in range(model.nc):
            if any(a == i or b == i for (a, b, _, _) in model.assoc):
                a_assoc = a_assoc + x[i] * (lnX[2 * i] + lnX[2 * i + 1])
    return rho_tot * (a_hc + a_disp + a_assoc)


def mu_res(model, rho, T):
    """Residual chemical potential mu_res / (k_B T) at (rho, T) -- the Clapeyron
    ``VT_chemical_potential_res / (R T)`` of PCSAFT.jl:69."""
    rho = np.asarray(rho, dtype=np.float64)
    out = np.zeros(len(rho))
    for i in range(len(rho)):
        h = 1e-30 * max(abs(rho[i]), 1.0)
        r = rho.astype(complex)
        r[i] += 1j * h
        out[i] = helmholtz_res_density(model, r, T).imag / (h * N_A)
    return out


def pressure(model, rho, T):
    """Bulk pressure in Pa from the Euler relation."""
    rho = np.asarray(rho, dtype=np.float64)
    f = helmholtz_res_density(model, rho, T).real
    mr = mu_res(model, rho, T)
    rho_n = rho * N_A
    return K_B * T * (np.sum(rho_n) + np.sum(rho_n * mr) - f)


def mu_total(model, rho, T):
    """Total chemical potential in J/mol, with the ideal part of the reference's
    BasicIdeal functional f_ideal = N_A n (ln n - 1.5 ln T - 1)
    (src/models/BasicIdeal.jl:34-38): mu_id/RT = ln(rho) - 1.5 ln T."""
    rho = np.asarray(rho, dtype=np.float64)
    return R_GAS * T * (np.log(rho) - 1.5 * np.log(T) + mu_res(model, rho, T))


def _dp_deta(model, x, T, eta):
    d = model.hs_diameter(T)
    scale = np.pi / 6.0 * np.sum(x * model.m * d ** 3) * N_A
    rho_tot = eta / scale
    return pressure(model, x * rho_tot, T), rho_tot


def density(model, p, T, x, phase="liquid", eta_guess=None):
    """Molar density (mol/m^3) at (p, T, x): liquid = largest root, vapour = smallest.

    Roots of p(eta) - p are bracketed on a coarse packing-fraction grid (or
    around ``eta_guess``) and polished with Brent's method."""
    from scipy.optimize import brentq
    x = np.asarray(x, dtype=np.float64)
    x = x / np.sum(x)

    def f(e):
        return _dp_deta(model, x, T, e)[0] - p

    if eta_guess is not None:
        a, b = eta_guess * 0.97, min(eta_guess * 1.03, 0.7405)
        fa, fb = f(a), f(b)
        if np.sign(fa) != np.sign(fb):
            eta = brentq(f, a, b, xtol=1e-17, rtol=1e-15, maxiter=200)
            return _dp_deta(model, x, T, eta)[1]
    etas = np.concatenate([np.logspace(-12, -1.3, 40), np.linspace(0.051, 0.74, 70)])
    vals = np.array([f(e) for e in etas])
    idx = np.nonzero(np.sign(vals[:-1]) != np.sign(vals[1:]))[0]
    if idx.size == 0:
        raise RuntimeError("no density root")
    k = idx[-1] if phase == "liquid" else idx[0]
    eta = brentq(f, etas[k], etas[k + 1], xtol=1e-17, rtol=1e-15, maxiter=200)
    return _dp_deta(model, x, T, eta)[1]


def volume(model, p, T, x, phase="liquid"):
    return 1.0 / density(model, p, T, x, phase)


def saturation_pure(model, T, p_guess=None):
    """Pure-component VLE at T: returns (p_sat, rho_liquid, rho_vapour) in (Pa, mol/m^3)."""
    if p_guess is None:
        p_guess = 1e3
    rl = density(model, p_guess, T, [1.0], "liquid")
    rv = p_guess / (R_GAS * T)
    y = np.log([rl, rv])
    for _ in range(100):
        def F(yy):
            a, b = np.exp(yy)
            return np.array([
                (pressure(model, [a], T) - pressure(model, [b], T)) / (R_GAS * T),
                (np.log(a) + mu_res(model, [a], T)[0]) - (np.log(b) + mu_res(model, [b], T)[0]),
            ])
        f0 = F(y)
        J = np.zeros((2, 2))
        for k in range(2):
            h = 1e-7
            yp = y.copy()
            yp[k] += h
            ym = y.copy()
            ym[k] -= h
            J[:, k] = (F(yp) - F(ym)) / (2 * h)
        step = np.linalg.solve(J, f0)
        lam = 1.0
        while np.max(np.abs(lam * step)) > 0.5:
            lam *= 0.5
        y = y - lam * step
        if np.max(np.abs(step)) < 1e-13:
            break
    rl, rv = np.exp(y)
    return float(pressure(model, [rl], T)), float(rl), float(rv)


def critical_temperature(model):
    """Pure-component critical temperature: the T where min_rho dp/drho == 0."""
    d0 = model.hs_diameter

    def min_dpdrho(T):
        scale = np.pi / 6.0 * model.m[0] * d0(T)[0] ** 3 * N_A
        best = np.inf
        for e in np.linspace(0.05, 0.35, 61):
            r = e / scale
            h = 1e-6 * r
            best = min(best, (pressure(model, [r + h], T) - pressure(model, [r - h], T)) / (2 * h))
        return best

    lo, hi = 50.0, 2000.0
    while min_dpdrho(lo) > 0:
        lo *= 0.7
    for _ in range(40):
        mid = 0.5 * (lo + hi)
        if min_dpdrho(mid) < 0:
            lo = mid
        else:
            hi = mid
    return 0.5 * (lo + hi)


def lle_binary(model, p, T, x_feed=(0.5, 0.5), guess=((0.999, 0.001), (0.001, 0.999)), iters=400):
    """Binary liquid--liquid equilibrium at (p, T) by K-value substitution
    (the ``tp_flash(..., RRTPFlash(equilibrium=:lle))`` of test/test_methods.jl).
    Returns (x1, x2) mole-fraction vectors of the two liquid phases."""
    x1 = np.array(guess[0], dtype=np.float64)
    x2 = np.array(guess[1], dtype=np.float64)

    eta_hint = {}

    def lnphi(x, key):
        r = density(model, p, T, x, "liquid", eta_hint.get(key))
        d = model.hs_diameter(T)
        eta_hint[key] = np.pi / 6 * np.sum(x / np.sum(x) * model.m * d ** 3) * N_A * r
        rho = r * x
        Z = p / (r * R_GAS * T)
        return mu_res(model, rho, T) - np.log(Z)

    z = np.asarray(x_feed, dtype=np.float64)
    for _ in range(iters):
        l1, l2 = lnphi(x1, 1), lnphi(x2, 2)
        K = np.exp(l1 - l2)  # x2_i = K_i x1_i
        a, b = 1e-12, 1 - 1e-12   # Rachford--Rice on the feed
        for _ in range(200):
            beta = 0.5 * (a + b)
            g = np.sum(z * (K - 1) / (1 + beta * (K - 1)))
            if g > 0:
                a = beta
            else:
                b = beta
        x1n = z / (1 + beta * (K - 1))
        x2n = K * x1n
        x1n /= np.sum(x1n)
        x2n /= np.sum(x2n)
        done = np.max(np.abs(np.log(x1n) - np.log(x1))) + np.max(np.abs(np.log(x2n) - np.log(x2))) < 1e-13
        x1, x2 = x1n, x2n
        if done:
            break
    return x1, x2
