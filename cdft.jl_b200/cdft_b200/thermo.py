"""Setup-time bulk PC-SAFT for the host API.

In the reference these numbers come from Clapeyron.jl (hard-sphere diameter
``d``, ``VT_chemical_potential_res``, ``volume``, ``bubble_pressure``,
``tp_flash``, ``crit_pure``; called from PCSAFT.jl:65-72, two_phase.jl:1-6 and
src/methods/*.jl).  They enter the hot path only as plain inputs of the C ABI
(species chemical potentials, bulk densities), so this module is ordinary
host code: vectorised NumPy, FP64, derivatives by complex step.

Equations: Gross & Sadowski, Ind. Eng. Chem. Res. 40 (2001) 1244 and
41 (2002) 5510 (2B association).
"""
import numpy as np

N_A = 6.02214076e23
K_B = 1.380649e-23
R = N_A * K_B

_A = np.array([
    [0.9105631445, -0.3084016918, -0.0906148351], [0.6361281449, 0.1860531159, 0.4527842806],
    [2.6861347891, -2.5030047259, 0.5962700728], [-26.547362491, 21.419793629, -1.7241829131],
    [97.759208784, -65.25588533, -4.1302112531], [-159.59154087, 83.318680481, 13.77663187],
    [91.297774084, -33.74692293, -8.6728470368]])
_B = np.array([
    [0.7240946941, -0.5755498075, 0.0976883116], [2.2382791861, 0.6995095521, -0.2557574982],
    [-4.0025849485, 3.892567339, -9.155856153], [-21.003576815, -17.215471648, 20.642075974],
    [26.855641363, 192.67226447, -38.804430052], [206.55133841, -161.82646165, 93.626774077],
    [-355.60235612, -165.20769346, -29.666905585]])


_TC_CACHE = {}


class PCSAFT:
    """PC-SAFT parameters of a (one-bead-per-component) mixture.

    Clapeyron's parameter database is not shipped, so parameters are explicit:
    ``m`` segments, ``sigma`` in Angstrom, ``epsilon`` in K, optional ``kij``
    and 2B association ``assoc = {component_index: (eps_AB_K, kappa_AB)}``.
    """

    def __init__(self, components, m, sigma, epsilon, kij=None, assoc=None, assoc_cross=None):
        self.components = list(components)
        self.m = np.asarray(m, dtype=float)
        self.sigma = np.asarray(sigma, dtype=float) * 1e-10
        self.epsilon = np.asarray(epsilon, dtype=float)
        nc = len(self.m)
        k = np.zeros((nc, nc)) if kij is None else np.asarray(kij, dtype=float)
        self.kij = k
        self.sigma_ij = (self.sigma[:, None] + self.sigma[None, :]) / 2
        self.eps_ij = np.sqrt(np.outer(self.epsilon, self.epsilon)) * (1 - k)
        self.assoc = dict(assoc or {})
        # cross-association {(i, j): (eps_AB_K, kappa_AB)}: site A of i with B of j and A of j
        # with B of i (two of the reference's pairs, assoc.jl:18-56)
        self.assoc_cross = {tuple(sorted(k)): tuple(v) for k, v in dict(assoc_cross or {}).items()}
        for (i, j) in self.assoc_cross:
            if i == j or i not in self.assoc or j not in self.assoc:
                raise ValueError("cross-association needs two distinct self-associating components")

    def __len__(self):
        return len(self.m)

    def pure(self, i):
        a = {0: self.assoc[i]} if i in self.assoc else None
        return PCSAFT([self.components[i]], [self.m[i]], [self.sigma[i] * 1e10], [self.epsilon[i]], assoc=a)

    def theta(self):
        """Model parameters theta = (sigma_k [A], eps_k/k_B [K], m_k) for k < nc, flattened."""
        return np.column_stack([self.sigma * 1e10, self.epsilon, self.m]).ravel()

    def with_theta(self, theta):
        """Copy of the model with parameters theta (layout of theta())."""
        t = np.asarray(theta, dtype=float).reshape(-1, 3)
        return PCSAFT(self.components, t[:, 2], t[:, 0], t[:, 1], kij=self.kij, assoc=self.assoc,
                      assoc_cross=self.assoc_cross)

    def assoc_pairs(self):
        """Site pairs (icomp, isite, jcomp, jsite, eps_AB, kappa_AB) in pack_assoc_params'
        order (assoc.jl:18-56): each associating component has sites A (0) and B (1) of the
        2B scheme; a self pair bonds A_i-B_i, a cross entry A_i-B_j and A_j-B_i."""
        pairs = [(i, 0, i, 1, e, k) for i, (e, k) in sorted(self.assoc.items())]
        for (i, j), (e, k) in sorted(self.assoc_cross.items()):
            pairs += [(i, 0, j, 1, e, k), (j, 0, i, 1, e, k)]
        return pairs

    def length_scale(self):
        return float(self.sigma_ij.max())

    def d(self, T):
        return self.sigma * (1 - 0.12 * np.exp(-3 * self.epsilon / T))

    # -- residual Helmholtz energy density / kT (1/m^3) --------------------------
    def _f_res(self, rho, T):
        rn = np.asarray(rho) * N_A
        tot = rn.sum()
        x = rn / tot
        d = self.d(T)
        z = [np.pi / 6 * (rn * self.m * d ** k).sum() for k in range(4)]
        e = z[3]
        ome = 1 - e
        ahs = (3 * z[1] * z[2] / ome + z[2] ** 3 / (e * ome ** 2) + (z[2] ** 3 / e ** 2 - z[0]) * np.log(ome)) / z[0]

        def gij(dd):
            return 1 / ome + dd * 3 * z[2] / ome ** 2 + dd ** 2 * 2 * z[2] ** 2 / ome ** 3

        mb = (x * self.m).sum()
        ahc = mb * ahs - (x * (self.m - 1) * np.log(gij(d / 2))).sum()
        c1, c2 = (mb - 1) / mb, (mb - 1) * (mb - 2) / mb ** 2
        pw = e ** np.arange(7)
        I1 = ((_A[:, 0] + c1 * _A[:, 1] + c2 * _A[:, 2]) * pw).sum()
        I2 = ((_B[:, 0] + c1 * _B[:, 1] + c2 * _B[:, 2]) * pw).sum()
        C1 = 1 / (1 + mb * (8 * e - 2 * e ** 2) / ome ** 4
                  + (1 - mb) * (20 * e - 27 * e ** 2 + 12 * e ** 3 - 2 * e ** 4) / (ome * (2 - e)) ** 2)
        xx = np.outer(x, x) * np.outer(self.m, self.m) * self.sigma_ij ** 3
        m2es3 = (xx * self.eps_ij / T).sum()
        m2e2s3 = (xx * (self.eps_ij / T) ** 2).sum()
        adisp = -2 * np.pi * tot * I1 * m2es3 - np.pi * tot * mb * C1 * I2 * m2e2s3
        aas = 0.0
        if self.assoc and not self.assoc_cross:
            for i, (eab, kab) in self.assoc.items():
                # self-associating 2B: X_A = X_B = X, X = 1/(1 + rho_i X Delta)
                D = self.sigma_ij[i, i] ** 3 * gij(d[i] / 2) * kab * (np.exp(eab / T) - 1)
                q = rn[i] * D
                X = 2 / (1 + np.sqrt(1 + 4 * q))
                aas = aas + x[i] * 2 * (np.log(X) - X / 2 + 0.5)
        elif self.assoc:
            aas = self._assoc_general(rn, x, d, gij, T)
        return tot * (ahc + adisp + aas)

    def _assoc_general(self, rn, x, d, gij, T):
        """Wertheim with several pairs: X_s = 1/(1 + sum_t rho_c(t) Delta_st X_t) by damped
        substitution and Newton (complex-step safe), a = sum_i x_i sum_a (ln X - X/2 + 1/2)."""
        pairs = self.assoc_pairs()
        sites = sorted({(p[0], p[1]) for p in pairs} | {(p[2], p[3]) for p in pairs})
        gi = {k: q for q, k in enumerate(sites)}
        ns = len(sites)
        dt = complex if np.iscomplexobj(rn) else float
        K = np.zeros((ns, ns), dtype=dt)   # K[s, t] = rho_c(t) Delta_st
        for (i, a, j, b, e, k) in pairs:
            dij = d[i] * d[j] / (d[i] + d[j])
            D = self.sigma_ij[i, j] ** 3 * gij(dij) * k * (np.exp(e / T) - 1)
            K[gi[(i, a)], gi[(j, b)]] += rn[j] * D
            K[gi[(j, b)], gi[(i, a)]] += rn[i] * D
        X = np.full(ns, 0.9, dtype=dt)
        for _ in range(5 * ns):
            X = 0.5 * (X + 1 / (1 + K @ X))
        for _ in range(12):
            C = K @ X
            J = np.diag(1 + C) + X[:, None] * K
            X = X - np.linalg.solve(J, X * (1 + C) - 1)
        return sum(x[c] * (np.log(X[q]) - X[q] / 2 + 0.5) for q, (c, _) in enumerate(sites))

    def mu_res(self, rho, T):
        """mu_res / kT of every component at molar densities ``rho``."""
        rho = np.asarray(rho, dtype=float)
        out = np.empty(len(rho))
        for i in range(len(rho)):
            h = 1e-30 * max(rho[i], 1.0)
            r = rho.astype(complex)
            r[i] += 1j * h
            out[i] = self._f_res(r, T).imag / (h * N_A)
        return out

    def pressure(self, rho, T):
        rho = np.asarray(rho, dtype=float)
        rn = rho * N_A
        return K_B * T * (rn.sum() + (rn * self.mu_res(rho, T)).sum() - self._f_res(rho, T).real)

    def chemical_potential(self, rho, T):
        """Total mu in J/mol, ideal part matching BasicIdeal (ln rho - 1.5 ln T)."""
        rho = np.asarray(rho, dtype=float)
        return R * T * (np.log(rho) - 1.5 * np.log(T) + self.mu_res(rho, T))

    def molar_density(self, p, T, x, phase="liquid", eta_guess=None):
        """Molar density at (p, T, x); liquid = densest root, vapour = most dilute."""
        from scipy.optimize import brentq
        x = np.asarray(x, dtype=float) / np.sum(x)
        scale = np.pi / 6 * (x * self.m * self.d(T) ** 3).sum() * N_A

        def f(eta):
            return self.pressure(x * eta / scale, T) - p

        if eta_guess is not None:
            a, b = 0.97 * eta_guess, min(1.03 * eta_guess, 0.7405)
            if (f(a) > 0) != (f(b) > 0):
                return brentq(f, a, b, xtol=1e-17, rtol=1e-15) / scale
        grid = np.concatenate([np.logspace(-12, -1.3, 40), np.linspace(0.051, 0.74, 70)])
        vals = np.array([f(g) for g in grid])
        idx = np.nonzero(np.sign(vals[:-1]) != np.sign(vals[1:]))[0]
        if idx.size == 0:
            raise ValueError("no density root at the given state")
        k = idx[-1] if phase == "liquid" else idx[0]
        return brentq(f, grid[k], grid[k + 1], xtol=1e-17, rtol=1e-15) / scale

    def stable_density(self, p, T, x):
        """Molar density of the stable phase at (p, T, x): of the vapour-like and
        liquid-like roots, the one with the lower Gibbs energy per mole
        (Clapeyron's volume(model, p, T, x) default)."""
        x = np.asarray(x, dtype=float) / np.sum(x)
        rl = self.molar_density(p, T, x, "liquid")
        rv = self.molar_density(p, T, x, "vapour")
        if abs(rl / rv - 1) < 1e-10:
            return rl
        g = [float((x * self.chemical_potential(x * r, T)).sum()) for r in (rl, rv)]
        return rl if g[0] <= g[1] else rv

    def volume(self, p, T, x, phase="liquid"):
        return 1.0 / self.molar_density(p, T, x, phase)

    def saturation(self, T, p0=1e3):
        """Pure-component VLE: (p_sat, rho_liquid, rho_vapour)."""
        y = np.log([self.molar_density(p0, T, [1.0], "liquid"), p0 / (R * T)])

        def F(v):
            a, b = np.exp(v)
            return np.array([(self.pressure([a], T) - self.pressure([b], T)) / (R * T),
                             np.log(a / b) + self.mu_res([a], T)[0] - self.mu_res([b], T)[0]])

        for _ in range(100):
            f0 = F(y)
            J = np.column_stack([(F(y + h) - F(y - h)) / 2e-7 for h in np.eye(2) * 1e-7])
            dy = np.linalg.solve(J, f0)
            dy *= min(1.0, 0.5 / np.max(np.abs(dy)))
            y = y - dy
            if np.max(np.abs(dy)) < 1e-13:
                break
        a, b = np.exp(y)
        return float(self.pressure([a], T)), float(a), float(b)

    def critical_temperature(self):
        """T at which the isotherm first has a horizontal inflection (pure component)."""
        key = (float(self.m[0]), float(self.sigma[0]), float(self.epsilon[0]), tuple(self.assoc.get(0, ())))
        if key in _TC_CACHE:
            return _TC_CACHE[key]

        def min_slope(T):
            scale = np.pi / 6 * self.m[0] * self.d(T)[0] ** 3 * N_A
            r = np.linspace(0.05, 0.35, 61) / scale
            return min((self.pressure([v * (1 + 1e-6)], T) - self.pressure([v * (1 - 1e-6)], T)) / (2e-6 * v) for v in r)

        lo, hi = 30.0, 3000.0
        while min_slope(lo) > 0:
            lo *= 0.7
        for _ in range(40):
            mid = 0.5 * (lo + hi)
            if min_slope(mid) < 0:
                lo = mid
            else:
                hi = mid
        _TC_CACHE[key] = 0.5 * (lo + hi)
        return _TC_CACHE[key]

    def lle(self, p, T, z=(0.5, 0.5), x1=(0.999, 0.001), x2=(0.001, 0.999), iters=400):
        """Binary liquid-liquid split at (p, T): K-value substitution + Rachford-Rice."""
        z = np.asarray(z, dtype=float)
        x1 = np.asarray(x1, dtype=float)
        x2 = np.asarray(x2, dtype=float)

        hint = {}

        def lnphi(x, key):
            r = self.molar_density(p, T, x, "liquid", hint.get(key))
            hint[key] = np.pi / 6 * (x / x.sum() * self.m * self.d(T) ** 3).sum() * N_A * r
            return self.mu_res(r * x, T) - np.log(p / (r * R * T))

        for _ in range(iters):
            K = np.exp(lnphi(x1, 1) - lnphi(x2, 2))
            lo, hi = 1e-12, 1 - 1e-12
            for _ in range(200):
                b = 0.5 * (lo + hi)
                if np.sum(z * (K - 1) / (1 + b * (K - 1))) > 0:
                    lo = b
                else:
                    hi = b
            n1 = z / (1 + b * (K - 1))
            n2 = K * n1
            n1, n2 = n1 / n1.sum(), n2 / n2.sum()
            done = np.max(np.abs(np.log(n1 / x1))) + np.max(np.abs(np.log(n2 / x2))) < 1e-14
            x1, x2 = n1, n2
            if done:
                break
        return x1, x2


def coexistence_sensitivity(model, T, rho1, rho2, p=None, rel=1e-6):
    """Derivatives of a two-phase bulk state with respect to theta = model.theta().

    Pure fluids (VLE): the unknowns (rho1, rho2) solve mu(rho1) = mu(rho2),
    p(rho1) = p(rho2); binaries at fixed (p, T) (LLE): mu_i(rho1) = mu_i(rho2),
    p(rho1) = p(rho2) = p.  The implicit-function theorem gives d rho / d theta;
    partial derivatives by central differences (relative step ``rel``).  Returns
    (dmu, dp): dmu[i, t] = d mu_i(rho1) / d theta_t in J/mol (total mu of
    chemical_potential, the one surface_tension uses) and dp[t] in Pa (zero at fixed p).
    """
    rho1 = np.asarray(rho1, dtype=float)
    rho2 = np.asarray(rho2, dtype=float)
    nc = len(model)
    if nc > 2:
        raise NotImplementedError("coexistence sensitivity for pure fluids and binaries")
    theta = model.theta()
    nt = theta.size
    x0 = np.concatenate([rho1, rho2])
    pscale = R * T * x0.max()

    def resid(x, mdl):
        a, b = x[:nc], x[nc:]
        mu = (mdl.chemical_potential(a, T) - mdl.chemical_potential(b, T)) / (R * T)
        pa, pb = mdl.pressure(a, T), mdl.pressure(b, T)
        if nc == 1:
            return np.concatenate([mu, [(pa - pb) / pscale]])
        return np.concatenate([mu, [(pa - p) / pscale, (pb - p) / pscale]])

    def dtheta(fun):
        cols = []
        for t in range(nt):
            h = rel * max(abs(theta[t]), 1.0)
            tp, tm = theta.copy(), theta.copy()
            tp[t] += h
            tm[t] -= h
            cols.append((np.asarray(fun(model.with_theta(tp))) - np.asarray(fun(model.with_theta(tm)))) / (2 * h))
        return np.column_stack(cols)

    J = np.empty((2 * nc, 2 * nc))
    for j in range(2 * nc):
        h = rel * x0[j]
        xp, xm = x0.copy(), x0.copy()
        xp[j] += h
        xm[j] -= h
        J[:, j] = (resid(xp, model) - resid(xm, model)) / (2 * h)
    dx = -np.linalg.solve(J, dtheta(lambda mdl: resid(x0, mdl)))
    d1 = dx[:nc]
    # total derivative of mu(rho1(theta); theta) and p(rho1(theta); theta)
    dmu = dtheta(lambda mdl: mdl.chemical_potential(rho1, T))
    dp = dtheta(lambda mdl: [mdl.pressure(rho1, T)])[0]
    Jmu = np.empty((nc, nc))
    Jp = np.empty(nc)
    for j in range(nc):
        h = rel * rho1[j]
        rp, rm = rho1.copy(), rho1.copy()
        rp[j] += h
        rm[j] -= h
        Jmu[:, j] = (model.chemical_potential(rp, T) - model.chemical_potential(rm, T)) / (2 * h)
        Jp[j] = (model.pressure(rp, T) - model.pressure(rm, T)) / (2 * h)
    dmu = dmu + Jmu @ d1
    dp = dp + Jp @ d1 if nc == 1 else np.zeros(nt)
    return dmu, dp
