"""PC-SAFT weighted-density functional on Cartesian grids (TEST ORACLE).

A NumPy FP64 restatement of the reference's converge! path:

* structures / grids  -- src/base/structure.jl:116-130,178-181,310-352;
  src/structure/structure.jl:138-195 (coords = LinRange(lb,ub,N); FFT frequencies
  fftfreq(N, N/(ub-lb)); Simpson spacing (ub-lb)/N)
* weighted-density kernels -- src/fields/weighted_densities.jl:28-80 (scalar) and
  :193-246 (vector); field list get_fields(::PCSAFTModel), PCSAFT.jl:47-62
* convolution -- src/utils/integrals.jl:88-96 (complex FFT, multiply, inverse, real)
* evaluate/integrate -- weighted_densities.jl:118-164 and :345-385, dispatcher
  src/fields/fields.jl:26-61 (rho field copied / overwrites, vector fields ``-=``)
* Phi = f_hs + f_hc + f_disp + f_assoc -- FMT.jl:17-46, PCSAFT.jl:110-211,
  assoc.jl:159-168,702-769 (analytic one-pair association) and :771-828 with
  _assoc_solve :405-413 (several pairs: 5 NS blended substitutions, 5 NS safeguarded
  Newton steps)
* dPhi/dn -- the reference differentiates with Enzyme forward mode
  (models.jl:377-389); here: complex-step forward derivatives, one per
  (field, component) direction, exact to rounding for these analytic expressions
* Steele wall -- src/structure/external_fields/steele.jl:31-81
* profile initialisation -- src/structure/structure.jl:50-93,125-136,
  external_field.jl:21-26, two_phase.jl:1-35
* get_new_profile! -- src/methods/converge.jl:108-153; converge! :220-254
* free energies, Simpson rule, gamma, adsorption -- models.jl:72-91,
  BasicIdeal.jl:10-38, utils/integrals.jl:17-41 (``_∫``), methods/surface_tension.jl:31-53,
  methods/adsorption.jl:16-32

Array layout: a profile is (nc, *grid) and weighted densities (nc, NF, *grid),
grid axes in reverse order (..., Nz, Ny, Nx) so the memory order is the
reference's Julia column-major (ngrid..., NF, nc) layout with x fastest.
"""
import numpy as np

from . import pcsaft_bulk as pb
from .anderson import aasol

N_A = pb.N_A
K_B = pb.K_B
PSI_DISP = 1.3862  # PCSAFT.jl:53,160

# field types
RHO, INT_DZ, INT_Z2DZ, INT_ZDZ = 0, 1, 2, 3


class SteeleWall:
    """Steele 10-4-3 wall (steele.jl:31-46); lengths in Angstrom as in the
    parameter database (database/Steele/steele_like.csv), converted to SI."""

    def __init__(self, sigma_A, eps_K, rho_A3, delta_A, width_m=0.0):
        self.sigma = sigma_A * 1e-10
        self.eps = eps_K
        self.rho = rho_A3 * 1e30
        self.delta = delta_A * 1e-10
        self.width = width_m

    @staticmethod
    def graphite(width_m=0.0):
        # graphite row of database/Steele/steele_like.csv: epsilon 28, sigma 3.4, rho 0.114, delta 3.35
        return SteeleWall(3.4, 28.0, 0.114, 3.35, width_m)


class Structure:
    """Cartesian structure: kind 'uniform' or 'twophase' (TwoPhase1DCart)."""

    def __init__(self, conditions, rho_bulk, bounds, ngrid, kind="uniform", rho_bulk2=None):
        self.p, self.T = float(conditions[0]), float(conditions[1])
        self.rho_bulk = np.asarray(rho_bulk, dtype=np.float64)
        self.bounds = [tuple(map(float, b)) for b in bounds]
        self.ngrid = tuple(int(n) for n in ngrid)
        self.kind = kind
        self.rho_bulk2 = None if rho_bulk2 is None else np.asarray(rho_bulk2, dtype=np.float64)

    @property
    def nd(self):
        return len(self.ngrid)

    @property
    def grid_shape(self):
        return tuple(reversed(self.ngrid))

    def coords(self, d):
        lb, ub = self.bounds[d]
        return np.linspace(lb, ub, self.ngrid[d])

    def dz(self):
        return [(ub - lb) / n for (lb, ub), n in zip(self.bounds, self.ngrid)]


def fftfreq(n, fs):
    # Julia's fftfreq(n, fs): [0, 1, ..., ceil(n/2)-1, -floor(n/2), ..., -1] * fs/n
    return np.fft.fftfreq(n) * fs


class DFTSystem:
    """PC-SAFT DFT system (base.jl:50-90 ``DFTSystem`` / ``build_DFT_system``)."""

    def __init__(self, model, structure, walls=None, vext=None):
        self.model = model
        self.structure = structure
        self.walls = list(walls or [])
        self._vext_given = None if vext is None else np.asarray(vext, dtype=np.float64)
        # True: the reference's literal White-Bear bracket (FMT.jl:39-45) everywhere,
        # including |n3| < 0.05 where the series form replaces it by default
        self.wb_closed = False
        T = structure.T
        self.nc = model.nc
        self.nd = structure.nd
        self.NF = 6 + self.nd
        self.L = model.length_scale()
        self.hsd = model.hs_diameter(T)              # m
        self.hsd_red = self.hsd / self.L            # PCSAFT.jl:221
        self.sigma_red = model.sigma_ij / self.L     # PCSAFT.jl:222
        self.eps_ij = model.eps_ij
        self.m = model.m
        # get_species: mu_res/RT at the bulk density of phase 1 (PCSAFT.jl:65-72)
        self.mu_res = pb.mu_res(model, structure.rho_bulk, T)
        self.chem_pot_res_dens = self.mu_res + np.log(structure.rho_bulk)  # converge.jl:121
        self.assoc_pairs = assoc_site_pairs(model)
        self.fields = self._field_list()
        self.kernels = self._build_kernels()
        self.vext = self._build_vext()

    # ---- fields (PCSAFT.jl:47-62) -------------------------------------------------
    def _field_list(self):
        d = self.hsd_red
        return [
            (RHO, np.zeros(self.nc)),
            (INT_DZ, 0.5 * d),
            (INT_Z2DZ, 0.5 * d),
            (INT_ZDZ, 0.5 * d),
            (INT_Z2DZ, d),
            (INT_DZ, d),
            (INT_Z2DZ, d * PSI_DISP),
        ]

    def _omega(self):
        s = self.structure
        comps = []
        for d in range(self.nd):
            lb, ub = s.bounds[d]
            w = fftfreq(s.ngrid[d], s.ngrid[d] / (ub - lb)) * self.L   # structure_fftfreq + _scaled_ω
            shape = [1] * self.nd
            shape[self.nd - 1 - d] = s.ngrid[d]
            comps.append(w.reshape(shape))
        return comps

    def _build_kernels(self):
        """Return a list over fields of arrays (nc, [nd,] *grid) (complex)."""
        om = self._omega()
        wbar = np.sqrt(sum(np.broadcast_to(o, self.structure.grid_shape) ** 2 for o in om))
        zero = wbar == 0
        safe = np.where(zero, 1.0, wbar)
        two_pi = 2 * np.pi
        out = []
        for ftype, width in self.fields:
            if ftype == RHO:
                out.append(None)
                continue
            per = []
            for i in range(self.nc):
                R = two_pi * width[i]
                if ftype == INT_DZ:
                    K = np.where(zero, 2 * R, 2 * np.sin(safe * R) / safe) / two_pi
                    per.append(K.astype(complex))
                elif ftype == INT_Z2DZ:
                    K = np.where(zero, 4 * np.pi * R ** 3 / 3,
                                 4 * np.pi / safe ** 3 * (np.sin(safe * R) - R * safe * np.cos(safe * R))) / two_pi ** 3
                    per.append(K.astype(complex))
                else:  # INT_ZDZ vector
                    comp = []
                    core = 4 * np.pi / safe ** 3 * (np.sin(safe * R) - R * safe * np.cos(safe * R))
                    for d in range(self.nd):
                        od = np.broadcast_to(om[d], self.structure.grid_shape)
                        K = np.where(zero, 4 * np.pi * 1j * R, 1j * od * core) / two_pi ** 3
                        comp.append(K)
                    per.append(np.stack(comp))
            out.append(np.stack(per))
        return out

    # ---- external field (steele.jl:49-81) ---------------------------------------
    def _build_vext(self):
        if self._vext_given is not None:
            return self._vext_given   # e.g. hard spherical solutes in 3D (no counterpart in the reference)
        if not self.walls:
            return None
        if self.nd != 1:
            raise NotImplementedError("Steele walls are restated for 1D Cartesian grids")
        z = self.structure.coords(0)
        T = self.structure.T
        V = np.zeros((self.nc, z.size))
        eps_i = self.model.eps
        sig_i = self.model.sigma
        for w in self.walls:
            eps_si = np.sqrt(w.eps * eps_i)
            sig_si = (w.sigma + sig_i) / 2
            for i in range(self.nc):
                s = sig_si[i]
                pre = 2 * np.pi * w.rho * eps_si[i] * w.delta * s ** 2
                V[i] += pre * (2 / 5 * (s / z) ** 10 - (s / z) ** 4 - s ** 4 / (3 * w.delta * (z + 0.61 * w.delta) ** 3))
                if w.width != 0:
                    hz = w.width - z
                    V[i] += pre * (2 / 5 * (s / hz) ** 10 - (s / hz) ** 4 - s ** 4 / (3 * w.delta * (hz + 0.61 * w.delta) ** 3))
        return V / T

    # ---- convolution (integrals.jl:88-96) ----------------------------------------
    def _conv(self, f, K):
        axes = tuple(range(-self.nd, 0))
        return np.real(np.fft.ifftn(np.fft.fftn(f, axes=axes) * K, axes=axes))

    def vector_slots(self):
        """Index ranges of the flattened field axis (field_indices, fields.jl:9-17)."""
        slots = []
        k = 0
        for ftype, _ in self.fields:
            ln = self.nd if ftype == INT_ZDZ else 1
            slots.append(range(k, k + ln))
            k += ln
        return slots

    def weighted_densities(self, rho):
        """evaluate_field! (fields.jl:26-48): n of shape (nc, NF, *grid)."""
        NA = N_A * self.L ** 3
        n = np.zeros((self.nc, self.NF) + self.structure.grid_shape)
        for (ftype, _), slot, K in zip(self.fields, self.vector_slots(), self.kernels):
            for i in range(self.nc):
                if ftype == RHO:
                    n[i, slot[0]] = rho[i] * NA
                elif ftype == INT_ZDZ:
                    for d in range(self.nd):
                        n[i, slot[d]] = self._conv(rho[i], K[i, d]) * NA
                else:
                    n[i, slot[0]] = self._conv(rho[i], K[i]) * NA
        return n

    def integrate(self, df):
        """integrate_field! (fields.jl:50-61): dF/drho_res of shape (nc, *grid)."""
        out = np.zeros((self.nc,) + self.structure.grid_shape)
        for (ftype, _), slot, K in zip(self.fields, self.vector_slots(), self.kernels):
            for i in range(self.nc):
                if ftype == RHO:
                    out[i] = df[i, slot[0]]
                elif ftype == INT_ZDZ:
                    for d in range(self.nd):
                        out[i] -= self._conv(df[i, slot[d]], K[i, d])
                else:
                    out[i] += self._conv(df[i, slot[0]], K[i])
        return out

    # ---- pointwise free-energy density ---------------------------------------------
    def phi(self, n):
        return f_res(n, self)

    def dphi(self, n):
        """dPhi/dn for every (component, field) direction, by complex step."""
        df = np.zeros(n.shape)
        base = n.astype(complex)
        for i in range(self.nc):
            for a in range(self.NF):
                h = np.maximum(1e-20 * np.abs(n[i, a]), 1e-250)
                pert = base.copy()
                pert[i, a] = pert[i, a] + 1j * h
                df[i, a] = f_res(pert, self).imag / h
        return df

    def dFdrho_res(self, rho):
        """δFδρ_res!(...) (models.jl:131-186) without the external field."""
        n = self.weighted_densities(rho)
        return self.integrate(self.dphi(n))

    def dFdrho(self, rho):
        """δFδρ_res(system, ρ) (models.jl:194-200): residual + external field."""
        out = self.dFdrho_res(rho)
        if self.vext is not None:
            out = out + self.vext
        return out

    def get_new_profile(self, rho):
        """converge.jl:108-153: ln G = (mu_res + ln rho_b) - dF/drho, clamped to +-100."""
        d = self.dFdrho(rho)
        lnG = self.chem_pot_res_dens.reshape((self.nc,) + (1,) * self.nd) - d
        return np.clip(lnG, -100.0, 100.0)

    # ---- dynamic DFT (ext/SciMLBasecDFTExt.jl:10-61) ---------------------------------
    def ddft_rhs(self, eta):
        """ddft_rhs_log! of SciMLBase.ODEProblem(system, ρ, tspan): with rho =
        exp(clamp(eta, -50, 30)) and mu = dF/drho_res + V_ext (δFδρ_res! then
        evaluate_external_field!), per component
        d eta = lap(eta) + lap(mu) + sum_d (grad_d eta)^2 + grad_d mu grad_d eta,
        each derivative the convolve! of the map 2 pi i k_d or -(2 pi)^2 |k|^2 (k = the
        reduced fftfreq grid, structure_ω * L) -- complex FFT, multiply, inverse, real part."""
        eta = np.asarray(eta, dtype=np.float64)
        rho = np.exp(np.clip(eta, -50.0, 30.0))
        mu = self.dFdrho(rho)
        om = [np.broadcast_to(o, self.structure.grid_shape) for o in self._omega()]
        lap = -(2 * np.pi) ** 2 * sum(o * o for o in om)
        grad = [2 * np.pi * 1j * o for o in om]
        out = np.zeros_like(eta)
        for i in range(self.nc):
            out[i] = self._conv(eta[i], lap) + self._conv(mu[i], lap)
            for g in grad:
                ge = self._conv(eta[i], g)
                out[i] += ge * ge + self._conv(mu[i], g) * ge
        return out

    # ---- profiles ----------------------------------------------------------------
    def initialize_profiles(self):
        s = self.structure
        rho = np.zeros((self.nc,) + s.grid_shape)
        if s.kind == "uniform":
            for i in range(self.nc):
                rho[i] = s.rho_bulk[i]
        elif s.kind == "twophase":
            # two_phase.jl:8-35 (periodic cos profile with two interfaces)
            lb, ub = s.bounds[0]
            H = ub - lb
            X = s.coords(0)
            for i in range(self.nc):
                Tc = pb.critical_temperature(self.model.split_pure(i))
                c0 = (2.4728 - 2.3625 * s.T / Tc) * (H / self.L)
                coef = np.sqrt(c0 ** 2 - 1) / 4
                rho[i] = cos_prof(X / (ub - lb), s.rho_bulk[i], s.rho_bulk2[i], ub / 4 + 3 * lb / 4, coef)
        else:
            raise ValueError(s.kind)
        if self.vext is not None:
            rho = rho * np.exp(-self.vext / 10)
        lo = np.finfo(np.float64).tiny ** (1 / 6)
        hi = np.finfo(np.float64).max ** (1 / 6)
        return np.clip(rho, lo, hi)

    # ---- integrals -----------------------------------------------------------------
    def integral(self, f):
        return simpson(f, self.structure)

    def F_res(self, rho):
        # models.jl:86-91
        n = self.weighted_densities(rho)
        return self.integral(self.phi(n)) / self.L ** 3

    def F_ideal(self, rho):
        # BasicIdeal.jl:10-38
        T = self.structure.T
        f = np.zeros(self.structure.grid_shape)
        for i in range(self.nc):
            f += N_A * rho[i] * (np.log(rho[i]) - 1.5 * np.log(T) - 1)
        return self.integral(f)

    def free_energy(self, rho):
        return self.F_ideal(rho) + self.F_res(rho)

    def surface_tension(self, rho):
        """surface_tension(system, ρ) (surface_tension.jl:31-53); the caller divides by 2."""
        s = self.structure
        F = self.free_energy(rho)
        mu = pb.mu_total(self.model, s.rho_bulk, s.T)
        chem = sum(mu[i] * self.integral(rho[i]) for i in range(self.nc))
        return F * K_B * s.T - chem + s.p * self.integral(np.ones(s.grid_shape))

    def adsorption(self, rho):
        V = np.prod([ub - lb for (lb, ub) in self.structure.bounds])
        return np.array([self.integral(rho[i]) / V for i in range(self.nc)])

    # ---- converge! -----------------------------------------------------------------
    def converge(self, rho0, maxit=10000, beta=1e-2, tol=1e-4, anderson_start=1e-1, anderson_m=5, callback=None):
        """converge!(prob, AASol(system; kw...), ρ), converge.jl:3-13,220-254."""
        shape = rho0.shape

        def gfix(lnx):
            rho = np.exp(lnx).reshape(shape)
            return self.get_new_profile(rho).ravel()

        out = aasol(gfix, np.log(rho0).ravel(), anderson_m, maxit=maxit, rtol=tol, atol=tol, beta=beta,
                    picard_maxit=maxit, picard_beta=beta, picard_rtol=anderson_start,
                    picard_atol=anderson_start, callback=callback)
        return np.exp(out.solution).reshape(shape), out


def cos_prof(x, start, stop, shift, coef):
    # src/structure/structure.jl:2
    c = np.cos((x - shift) * 2 * np.pi)
    return 0.5 * (start - stop) * c * np.sqrt((1 + coef ** 2) / (1 + coef ** 2 * c ** 2)) + 0.5 * (start + stop)


def simpson(f, structure):
    """``_∫`` (integrals.jl:17,28-41): coefficient 1 at both ends, 4 at even
    (1-based) interior indices, 2 at odd ones, times prod(dz/3), dz=(ub-lb)/N."""
    f = np.asarray(f)
    w = np.ones(())
    for ax, n in enumerate(f.shape):
        k = np.arange(1, n + 1)
        c = np.where((k == 1) | (k == n), 1.0, np.where(k % 2 == 0, 4.0, 2.0))
        shape = [1] * f.ndim
        shape[ax] = n
        w = w * c.reshape(shape)
    dz = structure.dz()
    return float(np.sum(w * f) * np.prod(np.array(dz) / 3))


def _logabs(z):
    # Base.log(abs(z)) with a complex-step-safe absolute value
    return np.log(z * np.sign(np.real(z)))


# Taylor coefficients of 12 pi B(n3), B the White-Bear bracket below: (j+1)(j+3)/(j+2)
_WB_SERIES = [(j + 1.0) * (j + 3.0) / (j + 2.0) for j in range(16)]
_WB_SMALL = 0.05


def _wb_bracket(n3, dn, log1dn, closed_only=False):
    """B(n3) = ln(1-n3)/(12 pi n3^2) + 1/(12 pi n3 (1-n3)^2) (FMT.jl:42-43).

    The closed form cancels from O(1/n3) to O(1) as n3 -> 0 (its derivative from
    O(1/n3^3)), which loses every digit where the kernels' ringing next to a hard
    solute takes n3 through zero; for |Re n3| < 0.05 the Taylor series
    12 pi B = sum_j (j+1)(j+3)/(j+2) n3^j (16 terms, FP64 rounding level there) is
    used instead.  Polynomial in n3, so the complex step differentiates it."""
    with np.errstate(all="ignore"):
        closed = log1dn / (12 * np.pi * n3 * n3) + 1.0 / (12 * np.pi * n3 * dn * dn)
    small = np.abs(np.real(n3)) < _WB_SMALL
    if closed_only or not np.any(small):
        return closed
    ser = _WB_SERIES[-1] + 0 * n3
    for c in _WB_SERIES[-2::-1]:
        ser = ser * n3 + c
    return np.where(small, ser / (12 * np.pi), closed)


def assoc_site_pairs(model):
    """Association site pairs as pack_assoc_params lays them out (assoc.jl:18-56):
    (icomp, isite, jcomp, jsite, eps_AB, kappa_AB, n_ia, n_jb).  Every associating
    component carries the two sites of the 2B scheme, A (0) and B (1), one of each; a
    model entry (i, j, eps, kappa) bonds A_i with B_j and, for i != j, A_j with B_i."""
    pairs = []
    for (i, j, eAB, kAB) in model.assoc:
        pairs.append((i, 0, j, 1, eAB, kAB, 1.0, 1.0))
        if i != j:
            pairs.append((j, 0, i, 1, eAB, kAB, 1.0, 1.0))
    return pairs


def _assoc_general(pairs, comp, deltas):
    """f_assoc with several pairs (assoc.jl:771-828): X_s of every site by _assoc_solve
    (:405-413) -- X0 = 0.9, 5 NS blended substitutions X <- (X + 1/(1 + C(X)))/2
    (:251-285), then 5 NS Newton steps on F = X (1 + C) - 1 whose candidate is kept where
    it lies in (0, 1) and replaced by the plain substitution elsewhere (:294-385) -- then
    sum_s u_c(s) n_s (ln X_s - X_s/2 + 1/2) with u_c = n0_c xi_c.  Complex-step safe: the
    derivative of the converged iteration is the implicit-function one the reference
    registers for Enzyme (:830-960)."""
    sites = []
    for (ic, ia, jc, jb, *_rest) in pairs:
        for key in ((ic, ia), (jc, jb)):
            if key not in sites:
                sites.append(key)
    sites.sort()
    NS = len(sites)
    gi = {k: q for q, k in enumerate(sites)}
    u = [n0 * xi for (n0, xi) in comp]
    # (site s, partner t, coefficient of X_t in C_s, component of t)
    terms = []
    for p, (ic, ia, jc, jb, _e, _k, nia, njb) in enumerate(pairs):
        sa, sb = gi[(ic, ia)], gi[(jc, jb)]
        terms.append((sa, sb, njb * u[jc] * deltas[p]))
        terms.append((sb, sa, nia * u[ic] * deltas[p]))
    mult = {}
    for (ic, ia, jc, jb, _e, _k, nia, njb) in pairs:
        mult[(ic, ia)] = nia
        mult[(jc, jb)] = njb
    shape = np.broadcast(*[t[2] for t in terms]).shape
    dt = complex if any(np.iscomplexobj(t[2]) for t in terms) else float
    X = [np.full(shape, 0.9, dtype=dt) for _ in range(NS)]

    def C_of(X):
        C = [np.zeros(shape, dtype=dt) for _ in range(NS)]
        for (s, t, kst) in terms:
            C[s] = C[s] + kst * X[t]
        return C

    for _ in range(5 * NS):
        C = C_of(X)
        X = [0.5 * (X[s] + 1.0 / (1.0 + C[s])) for s in range(NS)]
    for _ in range(5 * NS):
        C = C_of(X)
        ss = [1.0 / (1.0 + C[s]) for s in range(NS)]
        F = np.stack([X[s] * (1.0 + C[s]) - 1.0 for s in range(NS)], axis=-1)
        J = np.zeros(shape + (NS, NS), dtype=dt)
        for s in range(NS):
            J[..., s, s] = 1.0 + C[s]
        for (s, t, kst) in terms:
            J[..., s, t] = J[..., s, t] + X[s] * kst
        dX = np.linalg.solve(J, F[..., None])[..., 0]
        Xn = []
        for s in range(NS):
            cand = X[s] - dX[..., s]
            ok = (np.real(cand) > 0) & (np.real(cand) < 1)
            Xn.append(np.where(ok, cand, ss[s]))
        X = Xn
    res = 0.0
    for q, (c, a) in enumerate(sites):
        res = res + u[c] * mult[(c, a)] * (_logabs(X[q]) - 0.5 * X[q] + 0.5)
    return res


def f_res(n, sys):
    """Pointwise PC-SAFT residual free-energy density (PCSAFT.jl:110-117).

    ``n`` is (nc, NF, *grid), real or complex; returns (*grid)."""
    nc, nd = sys.nc, sys.nd
    m, d = sys.m, sys.hsd_red
    T = sys.structure.T
    F2, F3, FV = 1, 2, 3
    IHC, ILAM, IDISP = 3 + nd, 4 + nd, 5 + nd
    pi = np.pi
    # --- f_hs (FMT.jl:17-46) ---
    n0 = n1 = n2 = n3 = 0.0
    nv1 = [0.0] * nd
    nv2 = [0.0] * nd
    for i in range(nc):
        nim = n[i, F2] * m[i]
        n0 = n0 + nim / d[i]
        n1 = n1 + 0.5 * nim
        n2 = n2 + pi * nim * d[i]
        for k in range(nd):
            nvi = n[i, FV + k]
            nv1[k] = nv1[k] + nvi * m[i] / d[i]
            nv2[k] = nv2[k] - 2 * pi * nvi * m[i]
        n3 = n3 + n[i, F3] * m[i]
    nv1v2 = sum(nv1[k] * nv2[k] for k in range(nd))
    nv2sq = sum(nv2[k] * nv2[k] for k in range(nd))
    dn = 1.0 - n3
    log1dn = _logabs(dn)
    bkt = _wb_bracket(n3, dn, log1dn, getattr(sys, "wb_closed", False))
    res_hs = -n0 * log1dn + (n1 * n2 - nv1v2) / dn + (n2 * n2 * n2 / 3 - n2 * nv2sq) * bkt
    # --- f_hc (PCSAFT.jl:123-144) ---
    z3 = z2 = 0.0
    for i in range(nc):
        z3 = z3 + m[i] * n[i, IHC]
        z2 = z2 + m[i] * n[i, IHC] / d[i]
    z3 = z3 / 8
    z2 = z2 / 8
    inv1 = 1.0 / (1.0 - z3)
    res_hc = 0.0
    for i in range(nc):
        rhoi = n[i, 0]
        lam = n[i, ILAM] / (2 * d[i])
        ydd = inv1 + 1.5 * d[i] * z2 * inv1 * inv1 + 0.5 * d[i] * d[i] * z2 * z2 * inv1 ** 3
        res_hc = res_hc - rhoi * (m[i] - 1) * _logabs(ydd * lam / rhoi)
    # --- f_disp (PCSAFT.jl:150-197) ---
    psi = PSI_DISP
    factor = 3 / (4 * psi ** 3 * pi)
    rz = [n[i, IDISP] * factor / d[i] ** 3 for i in range(nc)]
    rz_sum = sum(rz)
    mbar = sum(rz[i] * m[i] for i in range(nc)) / rz_sum
    etad = sum(m[i] * rz[i] * d[i] ** 3 for i in range(nc)) * pi / 6
    s1 = s2 = 0.0
    for i in range(nc):
        for j in range(nc):
            cij = rz[i] * rz[j] * m[i] * m[j] * sys.sigma_red[i, j] ** 3
            eT = sys.eps_ij[i, j] / T
            s1 = s1 + cij * eT
            s2 = s2 + cij * eT * eT
    e2 = etad * etad
    C1 = (1 + mbar * (8 * etad - 2 * e2) / (1 - etad) ** 4
          + (1 - mbar) * (20 * etad - 27 * e2 + 12 * etad * e2 - 2 * e2 * e2) / ((1 - etad) ** 2 * (2 - etad) ** 2))
    c1 = (mbar - 1) / mbar
    c2 = c1 * (mbar - 2) / mbar
    I1 = 0.0
    I2 = 0.0
    for k in range(6, -1, -1):  # evalpoly (Horner)
        I1 = I1 * etad + (pb.PCSAFT_A[k, 0] + c1 * pb.PCSAFT_A[k, 1] + c2 * pb.PCSAFT_A[k, 2])
        I2 = I2 * etad + (pb.PCSAFT_B[k, 0] + c1 * pb.PCSAFT_B[k, 1] + c2 * pb.PCSAFT_B[k, 2])
    res_disp = -2 * (pi * I1 * s1) - pi * mbar * I2 * s2 / C1
    # --- f_assoc (assoc.jl:702-828) ---
    res_assoc = 0.0
    pairs = getattr(sys, "assoc_pairs", None) or assoc_site_pairs(sys.model)
    if pairs:
        n2m = 0.0
        n3m = 0.0
        for i in range(nc):
            n2m = n2m + pi * n[i, F2] * m[i] * d[i]
            n3m = n3m + n[i, F3] * m[i]
        nv2sqm = 0.0
        for k in range(nd):
            v = 0.0
            for i in range(nc):
                v = v - 2 * pi * n[i, FV + k] * m[i]
            nv2sqm = nv2sqm + v * v
        xim = 1.0 - nv2sqm / (n2m * n2m)
        inv1n3 = 1.0 / (1.0 - n3m)

        def delta_of(ic, jc, eAB, kAB):   # _assoc_delta, assoc.jl:159-168
            dij = d[ic] * d[jc] / (d[ic] + d[jc])
            ghs = inv1n3 + 0.5 * dij * xim * n2m * inv1n3 ** 2 + dij * dij * n2m * n2m * xim * inv1n3 ** 3 / 18
            return ghs * sys.sigma_red[ic, jc] ** 3 * (np.exp(eAB / T) - 1) * kAB

        def comp_terms(c):
            n0c = n[c, F2] / d[c]
            n2c = pi * n[c, F2] * d[c]
            sq = 0.0
            for k in range(nd):
                v = -2 * pi * n[c, FV + k]
                sq = sq + v * v
            return n0c, 1.0 - sq / (n2c * n2c)

        if len(pairs) == 1:   # analytic one-pair solution, assoc.jl:702-769
            ic, _, jc, _, eAB, kAB, nia, njb = pairs[0]
            delta = delta_of(ic, jc, eAB, kAB)
            n0i, xii = comp_terms(ic)
            n0j, xij = comp_terms(jc)
            kia = nia * n0i * xii * delta
            kjb = njb * n0j * xij * delta
            b = 1.0 - kia + kjb
            Xa = 2 / (b + np.sqrt(b * b + 4 * kia))
            Xb = 1.0 / (1.0 + kia * Xa)
            res_assoc = (n0i * xii * nia * (_logabs(Xa) - 0.5 * Xa + 0.5)
                         + n0j * xij * njb * (_logabs(Xb) - 0.5 * Xb + 0.5))
        else:
            res_assoc = _assoc_general(pairs, [comp_terms(c) for c in range(nc)],
                                       [delta_of(p[0], p[2], p[4], p[5]) for p in pairs])
    return res_hs + res_hc + res_disp + res_assoc
