"""Radial (spherical / cylindrical) restatement of the reference's QDHT path.

Test infrastructure only (the oracle).  Follows:

- `Uniform1DSphr` / `Uniform1DCyl` and `to_radial` (src/base/structure.jl:355-433): the
  grid is the QDHT sampling grid on [0, ub] (`Hankel.QDHT(0, 2, ub, N)` spherical,
  `Hankel.QDHT(0, 1, ub, N)` cylindrical);
- `SWeightedDensity(..., ::RadialFrequency)` (src/fields/weighted_densities.jl:92-116):
  the Cartesian closed forms at omega_bar = k / 2pi (scaled by L), no omega_bar = 0 branch;
  `evaluate_field!` / `integrate_field!` (:118-164): n = QDHT^-1[Omega * QDHT rho] N_A L^3,
  and the same convolution applied to dPhi/dn for the adjoint;
- `VWeightedDensity(..., ::RadialFrequency)` (:248-343): the dense operator
  T = D QDHT^-1 diag(H) QDHT with H the n3-type kernel at the *unscaled* omega_bar and
  physical width, D = `radial_derivative_matrix` (src/structure/transforms.jl:43-64);
  adjoint = the plain matrix transpose, added (`.+=`);
- the integral `4 pi integrateR` (sphere) / `2 pi integrateR` (cylinder)
  (src/utils/integrals.jl:15-19).

The QDHT itself comes from Hankel.jl (0.5.10), which is not vendored with the reference.
It is restated here from the published algorithm (M. Guizar-Sicairos and J. C.
Gutierrez-Vega, J. Opt. Soc. Am. A 21 (2004) 53): for the transform of a radially
symmetric function in D = n + 1 dimensions, order nu = (n - 1)/2 Bessel functions
(cylindrical n = 1: J_0; spherical n = 2: J_{1/2}, with r^{1/2}, k^{1/2} weights), zeros
j_1..j_{N+1}, S = j_{N+1}, r_m = j_m R / S, k_m = j_m / R, and the symmetric matrix
T_mn = 2 J_nu(j_m j_n / S) / (|J_{nu+1}(j_m)| |J_{nu+1}(j_n)| S), used for both directions.
In a forward-multiply-inverse convolution every constant factor cancels; what remains is
the sampling grid, the matrix and the per-point weights a_m = r_m^nu / |J_{nu+1}(j_m)|.
Parity of this restatement with Hankel.jl is pinned only by the bulk-consistency test of
the reference (test/test_coordinate_systems.jl:60-81, tolerance 1e-5).
"""
import numpy as np
from scipy import special

from . import functional as fn
from . import pcsaft_bulk as pb

N_A = pb.N_A


def bessel_zeros(nu, count):
    """First `count` positive zeros of J_nu (nu = 0 or 1/2)."""
    if nu == 0:
        return special.jn_zeros(0, count)
    if nu == 0.5:
        return np.pi * np.arange(1, count + 1, dtype=np.float64)
    raise ValueError(nu)


class QDHT:
    """Quasi-discrete Hankel transform on [0, R] with N points (see module docstring)."""

    def __init__(self, n, R, N):
        self.n = n
        self.nu = 0.0 if n == 1 else 0.5
        j = bessel_zeros(self.nu, N + 1)
        self.S = j[-1]
        self.j = j[:-1]
        self.R = float(R)
        self.N = N
        self.r = self.j * R / self.S
        self.k = self.j / R
        Jn1 = np.abs(special.jv(self.nu + 1, self.j))
        self.T = 2 * special.jv(self.nu, np.outer(self.j, self.j) / self.S) / (np.outer(Jn1, Jn1) * self.S)
        self.a = self.r ** self.nu / Jn1
        # integrateR: int_0^R f r^n dr (n = 2 nu + 1) by the Fourier-Bessel quadrature of
        # the k -> 0 limit: weights 2 R^2 / (S^2 J_{nu+1}(j_m)^2) r_m^(2 nu)
        # (nu = 1/2: exactly r_m^2 R / (N + 1) on the uniform grid r_m = m R / (N + 1))
        self.w = 2 * R ** 2 / (self.S ** 2 * Jn1 ** 2) * self.r ** (2 * self.nu)

    def conv_matrix(self, mult):
        """Dense operator f -> QDHT^-1[mult * QDHT f] on the sampling grid."""
        return (self.T * mult[None, :]) @ self.T * (self.a[None, :] / self.a[:, None])

    def integrate_r(self, f):
        return np.sum(self.w * f, axis=-1)


def radial_derivative_matrix(r):
    """transforms.jl:43-64: 2nd-order finite differences on a non-uniform grid."""
    N = len(r)
    D = np.zeros((N, N))
    for i in range(1, N - 1):
        h1, h2 = r[i] - r[i - 1], r[i + 1] - r[i]
        D[i, i - 1] = -h2 / (h1 * (h1 + h2))
        D[i, i] = (h2 - h1) / (h1 * h2)
        D[i, i + 1] = h1 / (h2 * (h1 + h2))
    h1, h2 = r[1] - r[0], r[2] - r[1]
    D[0, 0] = -(2 * h1 + h2) / (h1 * (h1 + h2))
    D[0, 1] = (h1 + h2) / (h1 * h2)
    D[0, 2] = -h1 / (h2 * (h1 + h2))
    h1, h2 = r[N - 2] - r[N - 3], r[N - 1] - r[N - 2]
    D[N - 1, N - 3] = h2 / (h1 * (h1 + h2))
    D[N - 1, N - 2] = -(h1 + h2) / (h1 * h2)
    D[N - 1, N - 1] = (2 * h2 + h1) / (h2 * (h1 + h2))
    return D


class RadialStructure(fn.Structure):
    """Uniform1DSphr / Uniform1DCyl: 1D radial grid = the QDHT sampling points on [0, ub];
    lb only places a Steele wall (structure.jl:365-433, steele.jl:111-143)."""

    def __init__(self, conditions, rho_bulk, ub, ngrid, coord, lb=0.0):
        super().__init__(conditions, rho_bulk, [(float(lb), ub)], (ngrid,), kind="uniform")
        self.coord = coord
        self.qdht = QDHT(2 if coord == "sphr" else 1, ub, ngrid)

    def coords(self, d=0):
        return self.qdht.r


class RadialDFTSystem(fn.DFTSystem):
    """The reference's PC-SAFT functional on a spherical or cylindrical grid."""

    def _build_kernels(self):
        Q = self.structure.qdht
        wbar = Q.k / (2 * np.pi) * self.L          # _scaled_omega (PCSAFT.jl:30-31)
        wraw = Q.k / (2 * np.pi)
        two_pi = 2 * np.pi
        D = radial_derivative_matrix(Q.r)
        out = []
        for ftype, width in self.fields:
            if ftype == fn.RHO:
                out.append(None)
                continue
            per = []
            for i in range(self.nc):
                if ftype == fn.INT_DZ:
                    R = two_pi * width[i]
                    per.append(Q.conv_matrix(2 * np.sin(wbar * R) / wbar / two_pi))
                elif ftype == fn.INT_Z2DZ:
                    R = two_pi * width[i]
                    per.append(Q.conv_matrix(4 * np.pi / wbar ** 3 * (np.sin(wbar * R) - R * wbar * np.cos(wbar * R))
                                             / two_pi ** 3))
                else:   # vector: D * (QDHT^-1 H QDHT), H at the raw omega and the physical width
                    Rk = two_pi * width[i] * self.L
                    H = 4 * np.pi / wraw ** 3 * (np.sin(wraw * Rk) - Rk * wraw * np.cos(wraw * Rk)) / two_pi ** 3
                    per.append(D @ Q.conv_matrix(H))
            out.append(np.stack(per))
        return out

    def _build_vext(self):
        """steele.jl:111-143: the planar single-wall Steele formula at the wall distance
        r - lb (lb > 0: fluid outside a solid sphere/cylinder) or ub - r (lb = 0: fluid in a
        pore of radius ub), clamped below at 0.5 min(sigma_i); the walls' widths play no part."""
        if self._vext_given is not None:
            return self._vext_given
        if not self.walls:
            return None
        r = self.structure.coords(0)
        lb, ub = self.structure.bounds[0]
        zw = np.maximum(r - lb if lb > 0 else ub - r, 0.5 * np.min(self.model.sigma))
        V = np.zeros((self.nc, r.size))
        for w in self.walls:
            eps_si = np.sqrt(w.eps * self.model.eps)
            sig_si = (w.sigma + self.model.sigma) / 2
            for i in range(self.nc):
                sg = sig_si[i]
                pre = 2 * np.pi * w.rho * eps_si[i] * w.delta * sg ** 2
                V[i] += pre * (2 / 5 * (sg / zw) ** 10 - (sg / zw) ** 4
                               - sg ** 4 / (3 * w.delta * (zw + 0.61 * w.delta) ** 3))
        return V / self.structure.T

    def weighted_densities(self, rho):
        NA = N_A * self.L ** 3
        n = np.zeros((self.nc, self.NF) + self.structure.grid_shape)
        for (ftype, _), slot, K in zip(self.fields, self.vector_slots(), self.kernels):
            for i in range(self.nc):
                if ftype == fn.RHO:
                    n[i, slot[0]] = rho[i] * NA
                else:
                    n[i, slot[0]] = (K[i] @ rho[i]) * NA
        return n

    def integrate(self, df):
        out = np.zeros((self.nc,) + self.structure.grid_shape)
        for (ftype, _), slot, K in zip(self.fields, self.vector_slots(), self.kernels):
            for i in range(self.nc):
                if ftype == fn.RHO:
                    out[i] = df[i, slot[0]]
                elif ftype == fn.INT_ZDZ:
                    out[i] += K[i].T @ df[i, slot[0]]
                else:
                    out[i] += K[i] @ df[i, slot[0]]
        return out

    def integral(self, f):
        ang = 4 * np.pi if self.structure.coord == "sphr" else 2 * np.pi
        return ang * self.structure.qdht.integrate_r(f)

    def adsorption(self, rho):
        ub = self.structure.bounds[0][1]
        V = 4 / 3 * np.pi * ub ** 3 if self.structure.coord == "sphr" else np.pi * ub ** 2
        return np.array([self.integral(rho[i]) / V for i in range(self.nc)])
