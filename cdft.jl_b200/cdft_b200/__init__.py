"""cdft_b200 -- B200-native converge! path of cDFT.jl behind the reference's API.

Host-side mirror of the reference's Julia interface for this path (same names,
argument meaning and error behaviour, Julia's ``!`` dropped):

    model     = PCSAFT([...], m=..., sigma=..., epsilon=...)       # Clapeyron model stand-in
    structure = Uniform1DCart((p, T), rho_bulk, [lb, ub], ngrid)   # src/base/structure.jl:310-352
    system    = DFTSystem(model, structure, Steele(["graphite"]))  # src/base/base.jl:75-90
    rho       = initialize_profiles(system)                        # src/structure/structure.jl:50-93
    converge(system, rho, beta=0.1, tol=1e-10, anderson_m=5)        # src/methods/converge.jl:214-254
    gamma     = surface_tension(system, rho)                       # src/methods/surface_tension.jl:31-53

Every compute call (dF/drho, F_res, converge) runs in libcdft_b200.so on the
GPU; importing this package raises if the library has not been built.
"""
import ctypes

import numpy as np

from . import _lib
from ._lib import CDFTError, PREC_FP64, PREC_MIXED
from .thermo import PCSAFT, N_A, K_B, R

_LIB = _lib.load()

__all__ = [
    "PCSAFT", "Steele", "HardSphereSolutes", "HardCore", "Uniform1DCart", "Uniform3DCart", "Uniform1DSphr",
    "Uniform1DCyl", "TwoPhase1DCart", "DFTOptions",
    "DFTSystem", "AASol",
    "initialize_profiles", "converge", "batch_converge", "dFdrho_res", "F_res", "F_ideal",
    "free_energy", "surface_tension", "interfacial_tension", "adsorption", "integrate", "ddft_rhs", "ddft_problem", "bulk_density",
    "F_res_grad", "grad_params", "dgamma_dtheta", "batch_integrals", "batch_properties", "grand_potential",
    "CDFTError", "launch_count", "tuning", "saturation",
]

PSI = 1.3862

# Steele parameter database row (database/Steele/steele_like.csv): epsilon K, sigma A, rho 1/A^3, delta A
_STEELE_DB = {"graphite": (28.0, 3.4, 0.114, 3.35)}


class Steele:
    """Steele 10-4-3 wall (src/structure/external_fields/steele.jl:31-46);
    ``width != 0`` adds a second wall at z = width (slit pore)."""

    def __init__(self, surface, width=0.0):
        self.surface = list(surface)
        for s in self.surface:
            if s not in _STEELE_DB:
                raise KeyError(f"Steele parameters for {s!r} are not in the database")
        eps, sig, rho, delta = (np.array([_STEELE_DB[s][k] for s in self.surface]) for k in range(4))
        self.epsilon = eps
        self.sigma = sig * 1e-10
        self.rho = rho * 1e30
        self.delta = delta * 1e-10
        self.width = float(width)

    def potential(self, model, z, T):
        """V_ext / k_B T on coordinates z for every component (steele.jl:49-81)."""
        nc = len(model)
        V = np.zeros((nc, z.size))
        for s in range(len(self.surface)):
            eps_si = np.sqrt(self.epsilon[s] * model.epsilon)
            sig_si = (self.sigma[s] + model.sigma) / 2
            for i in range(nc):
                sg = sig_si[i]
                pre = 2 * np.pi * self.rho[s] * eps_si[i] * self.delta[s] * sg ** 2
                for zz in ([z] if self.width == 0 else [z, self.width - z]):
                    V[i] += pre * (0.4 * (sg / zz) ** 10 - (sg / zz) ** 4
                                   - sg ** 4 / (3 * self.delta[s] * (zz + 0.61 * self.delta[s]) ** 3))
        return V / T

    def potential_dtheta(self, model, z, T):
        """d(V_i / k_B T)/d theta_t on coordinates z, shape (3 nc, nc, N), theta = (sigma_k [A],
        eps_k/k_B [K], m_k): V_i depends on its own component's parameters through
        sigma_si = (sigma_s + sigma_i)/2 and eps_si = sqrt(eps_s eps_i) (steele.jl:36-41,49-81)."""
        nc = len(model)
        out = np.zeros((3 * nc, nc, z.size))
        for s in range(len(self.surface)):
            eps_si = np.sqrt(self.epsilon[s] * model.epsilon)
            sig_si = (self.sigma[s] + model.sigma) / 2
            d = self.delta[s]
            for i in range(nc):
                sg = sig_si[i]
                pre = 2 * np.pi * self.rho[s] * eps_si[i] * d
                for zz in ([z] if self.width == 0 else [z, self.width - z]):
                    # V = pre A(sg) / T, A = 0.4 sg^12 z^-10 - sg^6 z^-4 - sg^6 / (3 d (z + 0.61 d)^3)
                    A = 0.4 * sg ** 12 / zz ** 10 - sg ** 6 / zz ** 4 - sg ** 6 / (3 * d * (zz + 0.61 * d) ** 3)
                    dA = 4.8 * sg ** 11 / zz ** 10 - 6 * sg ** 5 / zz ** 4 - 6 * sg ** 5 / (3 * d * (zz + 0.61 * d) ** 3)
                    out[3 * i + 0, i] += pre * dA * 0.5e-10 / T          # per Angstrom of sigma_i
                    out[3 * i + 1, i] += pre * A / T / (2 * model.epsilon[i])
        return out

    def potential_radial(self, model, r, T, lb, ub):
        """V_ext / k_B T on a spherical or cylindrical grid (steele.jl:111-143): the planar
        single-wall formula at the wall distance r - lb when lb > 0 (fluid outside a solid
        sphere or cylinder of radius lb), ub - r otherwise (fluid inside a pore of radius
        ub), clamped below at half the smallest fluid sigma; no second wall."""
        nc = len(model)
        r = np.asarray(r, dtype=float)
        zw = np.maximum(r - lb if lb > 0 else ub - r, 0.5 * np.min(model.sigma))
        V = np.zeros((nc, r.size))
        for s in range(len(self.surface)):
            eps_si = np.sqrt(self.epsilon[s] * model.epsilon)
            sig_si = (self.sigma[s] + model.sigma) / 2
            for i in range(nc):
                sg = sig_si[i]
                pre = 2 * np.pi * self.rho[s] * eps_si[i] * self.delta[s] * sg ** 2
                V[i] += pre * (0.4 * (sg / zw) ** 10 - (sg / zw) ** 4
                               - sg ** 4 / (3 * self.delta[s] * (zw + 0.61 * self.delta[s]) ** 3))
        return V / T


class HardSphereSolutes:
    """Hard spherical solutes in a periodic box (an external field the reference does
    not have; defined here for the 3D configuration): V_ext = `height` k_B T for fluid
    centres closer than `radius` to a solute centre (minimum image), 0 elsewhere.
    The height only has to saturate the clamp of ln G (converge.jl:150)."""

    def __init__(self, centres, radius, height=100.0):
        self.centres = np.asarray(centres, dtype=float).reshape(-1, 3)
        self.radius = float(radius)
        self.height = float(height)

    @staticmethod
    def seeded(n, radius, box, min_gap, seed=0):
        """n non-overlapping centres in [0, box)^3 by rejection sampling with
        numpy.random.default_rng(seed); centre distances >= 2 radius + min_gap."""
        rng = np.random.default_rng(seed)
        pts = []
        while len(pts) < n:
            c = rng.random(3) * box
            ok = True
            for q in pts:
                dv = c - q
                dv -= box * np.round(dv / box)
                if np.sqrt(dv @ dv) < 2 * radius + min_gap:
                    ok = False
                    break
            if ok:
                pts.append(c)
        return np.array(pts)

    def potential(self, model, structure):
        coords = [structure.coords(d) for d in range(3)]
        X, Y, Z = coords[0][None, None, :], coords[1][None, :, None], coords[2][:, None, None]
        box = [ub - lb for (lb, ub) in structure.bounds]
        inside = np.zeros(structure.grid_shape, dtype=bool)
        for c in self.centres:
            dx = X - c[0]
            dx = dx - box[0] * np.round(dx / box[0])
            dy = Y - c[1]
            dy = dy - box[1] * np.round(dy / box[1])
            dz = Z - c[2]
            dz = dz - box[2] * np.round(dz / box[2])
            inside |= dx * dx + dy * dy + dz * dz < self.radius ** 2
        V = np.where(inside, self.height, 0.0)
        return np.repeat(V[None], len(model), axis=0)


class Structure:
    coord = "cart"

    def __init__(self, conditions, rho_bulk, bounds, ngrid, kind, rho_bulk2=None):
        self.conditions = (float(conditions[0]), float(conditions[1]))
        self.rho_bulk = np.asarray(rho_bulk, dtype=float)
        b = np.asarray(bounds, dtype=float).reshape(-1, 2)
        self.bounds = [tuple(r) for r in b]
        ng = ngrid if isinstance(ngrid, (tuple, list)) else (ngrid,)
        self.ngrid = tuple(int(n) for n in ng)
        if len(self.ngrid) != len(self.bounds):
            raise ValueError("bounds and ngrid dimensions differ")
        self.kind = kind
        self.rho_bulk2 = None if rho_bulk2 is None else np.asarray(rho_bulk2, dtype=float)

    @property
    def nd(self):
        return len(self.ngrid)

    @property
    def grid_shape(self):
        return tuple(reversed(self.ngrid))   # (..., Nz, Ny, Nx): memory order of Julia's (Nx, Ny, Nz)

    def coords(self, d=0):
        lb, ub = self.bounds[d]
        return np.linspace(lb, ub, self.ngrid[d])   # LinRange(lb, ub, N)

    def dz(self):
        return [(ub - lb) / n for (lb, ub), n in zip(self.bounds, self.ngrid)]   # structure_dz


def Uniform1DCart(conditions, rho_bulk, bounds, ngrid):
    """src/base/structure.jl:310-312"""
    return Structure(conditions, rho_bulk, bounds, ngrid, "uniform")


def Uniform3DCart(conditions, rho_bulk, bounds, ngrid):
    """src/base/structure.jl:352 (cubic periodic boxes with N in {32, 64, 128, 256} on the GPU)."""
    b = np.asarray(bounds, dtype=float)
    if b.size == 2:
        b = np.tile(b.reshape(1, 2), (3, 1))
    ng = ngrid if isinstance(ngrid, (tuple, list)) else (ngrid,) * 3
    return Structure(conditions, rho_bulk, b, ng, "uniform")


class RadialStructure(Structure):
    """Uniform1DSphr / Uniform1DCyl (src/base/structure.jl:355-433): the grid is the
    sampling grid of the quasi-discrete Hankel transform on [0, ub] (the reference's
    Hankel.QDHT(0, n, ub, N), n = 2 sphere, 1 cylinder): r_m = j_m ub / j_{N+1} with j_m the
    zeros of J_nu, nu = 1/2 (sphere) or 0 (cylinder).  lb is kept for external fields."""

    def __init__(self, conditions, rho_bulk, bounds, ngrid, coord):
        b = np.asarray(bounds, dtype=float).ravel()
        if b.size == 1:
            b = np.array([0.0, b[0]])
        super().__init__(conditions, rho_bulk, b, ngrid, "uniform")
        self.coord = coord
        N = self.ngrid[0]
        ub = self.bounds[0][1]
        nu = 0.5 if coord == "sphr" else 0.0
        from scipy import special
        j = np.pi * np.arange(1, N + 2) if nu == 0.5 else special.jn_zeros(0, N + 1)
        S = j[-1]
        self._r = j[:-1] * ub / S
        jn1 = np.abs(special.jv(nu + 1, j[:-1]))
        ang = 4 * np.pi if coord == "sphr" else 2 * np.pi
        # 4 pi / 2 pi integrateR: Fourier-Bessel quadrature of int f r^(2 nu + 1) dr
        self.weights = ang * 2 * ub ** 2 / (S ** 2 * jn1 ** 2) * self._r ** (2 * nu)

    def coords(self, d=0):
        return self._r

    def volume(self):
        ub = self.bounds[0][1]
        return 4 / 3 * np.pi * ub ** 3 if self.coord == "sphr" else np.pi * ub ** 2


def Uniform1DSphr(conditions, rho_bulk, bounds, ngrid):
    """src/base/structure.jl:383 (spherical symmetry, radial grid on [0, ub])."""
    return RadialStructure(conditions, rho_bulk, bounds, ngrid, "sphr")


def Uniform1DCyl(conditions, rho_bulk, bounds, ngrid):
    """src/base/structure.jl:406 (cylindrical symmetry, radial grid on [0, ub])."""
    return RadialStructure(conditions, rho_bulk, bounds, ngrid, "cyl")


class HardCore:
    """A hard core of radius `radius` at the origin of a spherical or cylindrical grid
    (a solute or a rod): V_ext = `height` k_B T for r < radius.  An external field the
    reference does not define; it gives the radial systems structure to converge."""

    def __init__(self, radius, height=100.0):
        self.radius = float(radius)
        self.height = float(height)

    def potential(self, model, r, T):
        V = np.where(np.asarray(r) < self.radius, self.height, 0.0)
        return np.repeat(V[None], len(model), axis=0)


def TwoPhase1DCart(conditions, rho_bulk, rho_bulk2, bounds, ngrid):
    """src/base/structure.jl:487 (periodic cos seed with two interfaces, two_phase.jl:8-35)"""
    return Structure(conditions, rho_bulk, bounds, ngrid, "twophase", rho_bulk2)


class DFTOptions:
    """src/base/devices.jl:29-40: ``precision`` is "fp64" (Float64) or "mixed"
    (FP32 convolutions and Phi, FP64 solver and integrals, an FP64 polish).  The
    reference's Float32 runs everything in FP32; the library has no FP32 solver, so
    float32 is refused rather than mapped onto "mixed"."""

    def __init__(self, precision="fp64"):
        if precision in ("fp64", np.float64, float):
            self.precision = PREC_FP64
        elif precision == "mixed":
            self.precision = PREC_MIXED
        elif precision in ("fp32", np.float32):
            raise ValueError('precision float32 (all-FP32) is not offered: use "fp64" or "mixed"')
        else:
            raise ValueError(f"unknown precision {precision!r}")


class DFTSystem:
    """src/base/base.jl:50-90: model, species (get_species, PCSAFT.jl:65-72),
    structure, external fields and options; owns one device plan."""

    def __init__(self, model, structure, external_field=None, options=None):
        if structure.nd not in (1, 3):
            raise NotImplementedError("1D and 3D Cartesian structures are supported")
        self.model = model
        self.structure = structure
        if external_field is None:
            self.external_field = []
        elif isinstance(external_field, (list, tuple)):
            self.external_field = list(external_field)
        else:
            self.external_field = [external_field]
        self.options = options or DFTOptions()
        p, T = structure.conditions
        self.L = model.length_scale()
        self.size = model.d(T)                                   # species.size
        self.chempot_res = model.mu_res(structure.rho_bulk, T)   # species.chempot_res
        nc = len(model)
        nd = structure.nd
        self.vext = None
        if self.external_field:
            if nd == 1 and structure.coord != "cart":
                r = structure.coords(0)
                lb, ub = structure.bounds[0]
                self.vext = sum(f.potential_radial(model, r, T, lb, ub) if isinstance(f, Steele)
                                else f.potential(model, r, T) for f in self.external_field)
            elif nd == 1:
                z = structure.coords(0)
                self.vext = sum(f.potential(model, z, T) for f in self.external_field)
            else:
                self.vext = sum(f.potential(model, structure) for f in self.external_field)
        d = _lib.SystemDesc()
        d.nd = nd
        for k in range(nd):
            d.ngrid[k] = structure.ngrid[k]
            d.bounds[k][0], d.bounds[k][1] = structure.bounds[k]
        d.coord = {"cart": _lib.COORD_CART, "sphr": _lib.COORD_SPH, "cyl": _lib.COORD_CYL}[structure.coord]
        d.nc = nc
        for i in range(nc):
            d.m[i] = model.m[i]
            d.hsd[i] = self.size[i]
            d.mu_res_plus_ln_rhob[i] = self.chempot_res[i] + np.log(structure.rho_bulk[i])
            for j in range(nc):
                d.sigma[i * nc + j] = model.sigma_ij[i, j]
                d.eps[i * nc + j] = model.eps_ij[i, j]
        d.L = self.L
        d.T = T
        pairs = model.assoc_pairs()
        if len(pairs) > _lib.MAX_ASSOC:
            raise NotImplementedError(f"at most {_lib.MAX_ASSOC} association pairs per system")
        d.n_assoc = len(pairs)
        for q, (i, a, j, b, eab, kab) in enumerate(pairs):
            d.assoc[q] = _lib.AssocPair(i, j, a, b, 1, 1, eab, kab)
        self._vext_buf = None
        if self.vext is not None:
            self._vext_buf = np.ascontiguousarray(self.vext, dtype=np.float64)
            d.vext = _lib.dptr(self._vext_buf)
        d.precision = self.options.precision
        self._desc = d
        plan = ctypes.c_void_p()
        _lib.check(_LIB.cdft_plan_create(ctypes.byref(d), ctypes.byref(plan)))
        self._plan = plan

    @property
    def nc(self):
        return len(self.model)

    @property
    def ngrid(self):
        return self.structure.ngrid

    def close(self):
        if getattr(self, "_plan", None):
            _LIB.cdft_plan_destroy(self._plan)
            self._plan = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _cos_prof(x, start, stop, shift, coef):
    # src/structure/structure.jl:2
    c = np.cos((x - shift) * 2 * np.pi)
    return 0.5 * (start - stop) * c * np.sqrt((1 + coef ** 2) / (1 + coef ** 2 * c ** 2)) + 0.5 * (start + stop)


def initialize_profiles(system, noise=0.0, rng=None):
    """src/structure/structure.jl:50-93 (+ two_phase.jl:8-35, external_field.jl:21-26).
    Returns rho with shape (nc, N) -- the memory order of the reference's (N, nc)."""
    s = system.structure
    p, T = s.conditions
    nc = system.nc
    rho = np.empty((nc,) + s.grid_shape)
    if s.kind == "uniform":
        rho[:] = s.rho_bulk.reshape((nc,) + (1,) * s.nd)
    else:
        lb, ub = s.bounds[0]
        H = ub - lb
        X = s.coords(0)
        for i in range(nc):
            Tc = system.model.pure(i).critical_temperature()
            c0 = (2.4728 - 2.3625 * T / Tc) * (H / system.L)
            coef = np.sqrt(c0 ** 2 - 1) / 4
            rho[i] = _cos_prof(X / (ub - lb), s.rho_bulk[i], s.rho_bulk2[i], ub / 4 + 3 * lb / 4, coef)
    if system.vext is not None:
        rho *= np.exp(-system.vext / 10)
    if noise:
        rng = rng or np.random.default_rng()
        tot = rho.sum(axis=0)
        rho *= 1 + noise * (2 * rng.random(rho.shape) - 1)
        rho *= tot / rho.sum(axis=0)
    lo = np.finfo(np.float64).tiny ** (1 / 6)
    hi = np.finfo(np.float64).max ** (1 / 6)
    return np.clip(rho, lo, hi)


class AASol:
    """src/utils/anderson.jl:193-275 (solver options of aasol)."""

    def __init__(self, m=5, maxit=20, rtol=1e-10, atol=1e-10, beta=1.0, picard_maxit=0, picard_beta=1.0,
                 picard_rtol=1e-2, picard_atol=1e-2, verbose=False):
        if m < 0:
            raise ValueError("m must be >= 0")
        if not (0 < abs(beta) <= 1):
            raise ValueError("abs(beta) must be in (0,1]")
        self.m, self.maxit, self.rtol, self.atol, self.beta = m, maxit, rtol, atol, beta
        self.picard_maxit, self.picard_beta = picard_maxit, picard_beta
        self.picard_rtol, self.picard_atol = picard_rtol, picard_atol
        self.verbose = verbose

    @classmethod
    def for_system(cls, system=None, maxit=10000, beta=1e-2, tol=1e-4, anderson_start=1e-1, anderson_m=5,
                   verbose=False):
        """AASol(system; kwargs...) -> __AASol (converge.jl:3-12)."""
        return cls(anderson_m, maxit=maxit, rtol=tol, atol=tol, beta=beta, picard_maxit=maxit, picard_beta=beta,
                   picard_rtol=anderson_start, picard_atol=anderson_start, verbose=verbose)

    def c_opts(self, time_budget_s=0.0, iters_per_launch=0, engine="auto", mixed_switch_rtol=0.0):
        o = _lib.SolverOpts()
        o.m, o.maxit, o.rtol, o.atol, o.beta = self.m, self.maxit, self.rtol, self.atol, self.beta
        o.picard_maxit, o.picard_beta = self.picard_maxit, self.picard_beta
        o.picard_rtol, o.picard_atol = self.picard_rtol, self.picard_atol
        o.time_budget_s = time_budget_s
        o.iters_per_launch = iters_per_launch
        o.engine = {"auto": _lib.ENGINE_AUTO, "grid": _lib.ENGINE_GRID, "persistent": _lib.ENGINE_PERSISTENT}[engine]
        o.mixed_switch_rtol = mixed_switch_rtol
        return o


class ConvergeResult:
    def __init__(self, r, history):
        self.idid = bool(r.idid)
        self.errcode = r.errcode
        self.iterations = r.iterations
        self.evaluations = r.evaluations
        self.resnorm = r.resnorm
        self.tol = r.tol
        self.history = history

    def __repr__(self):
        return (f"ConvergeResult(idid={self.idid}, errcode={self.errcode}, iterations={self.iterations}, "
                f"evaluations={self.evaluations}, resnorm={self.resnorm:.3e})")


def _check_rho(system, rho):
    if not isinstance(rho, np.ndarray) or rho.dtype != np.float64 or not rho.flags["C_CONTIGUOUS"]:
        raise TypeError("rho must be a C-contiguous float64 numpy array")
    if rho.shape != (system.nc,) + tuple(reversed(system.ngrid)):
        raise ValueError(f"rho has shape {rho.shape}, expected {(system.nc,) + tuple(reversed(system.ngrid))}")


def converge(system, rho, method=None, time_budget_s=0.0, iters_per_launch=0, keep_history=True, engine="auto",
             mixed_switch_rtol=0.0, log_interval=0, save_interval=0, save_callback=None, **kwargs):
    """converge!(system, ρ; kwargs...) / converge!(system, ρ, solver): converges
    ``rho`` in place (converge.jl:214-254) and returns the aasol status.
    ``engine``: "auto", "grid" (per-stage kernels) or "persistent" (one CTA per system).
    ``save_interval`` / ``save_callback(it, rho)`` and ``log_interval`` are DFTProblem's
    hooks (converge.jl:31-60,256-267): the profile after every ``save_interval``
    evaluations goes to the callback, and the free energy of every ``log_interval``-th
    profile is logged (computed once converge returns: the callback runs while the plan is
    busy)."""
    _check_rho(system, rho)
    method = method or AASol.for_system(system, **kwargs)
    if save_interval > 0 and save_callback is None:
        raise ValueError("save_interval > 0 needs a save_callback")
    res = _lib.Result()
    hist = None
    if keep_history:
        cap = 2 * (method.maxit + 2 * method.picard_maxit + 4)
        hist = np.zeros(cap)
        res.history = _lib.dptr(hist)
        res.history_cap = cap
    opts = method.c_opts(time_budget_s, iters_per_launch, engine, mixed_switch_rtol)
    every = int(np.gcd(log_interval, save_interval)) if (log_interval and save_interval) else (log_interval or save_interval)
    logged = []
    if every > 0:
        shape = rho.shape

        def on_snapshot(user, s, it, ptr):
            prof = np.ctypeslib.as_array(ptr, shape=(rho.size,)).reshape(shape).copy()
            if save_interval and it % save_interval == 0:
                save_callback(it, prof)
            if log_interval and it % log_interval == 0:
                logged.append((it, prof))

        cb = _lib.SNAPSHOT_FN(on_snapshot)
        opts.snapshot_every = every
        opts.snapshot = ctypes.cast(cb, ctypes.c_void_p)
    _lib.check(_LIB.cdft_converge(system._plan, _lib.dptr(rho), ctypes.byref(opts), ctypes.byref(res)))
    for it, prof in logged:
        print(f"DFT iter {it:5d} | F = {free_energy(system, prof):.6g}")
    out = ConvergeResult(res, None if hist is None else hist[: res.history_len].copy())
    if method.verbose:
        msg = "DFT converged" if out.idid else "DFT did not converge"
        print(f"{msg} after {out.evaluations} evaluations: err = {out.resnorm:.3g}")
    return out


def batch_converge(systems, rhos, method=None, time_budget_s=0.0, iters_per_launch=0, engine="auto",
                   mixed_switch_rtol=0.0, **kwargs):
    """Converge many independent systems (state points, pore widths) together."""
    n = len(systems)
    if n != len(rhos):
        raise ValueError("systems and rhos differ in length")
    for s, r in zip(systems, rhos):
        _check_rho(s, r)
    method = method or AASol.for_system(systems[0], **kwargs)
    plans = (ctypes.c_void_p * n)(*[s._plan.value for s in systems])
    ptrs = (ctypes.POINTER(ctypes.c_double) * n)(*[_lib.dptr(r) for r in rhos])
    res = (_lib.Result * n)()
    opts = method.c_opts(time_budget_s, iters_per_launch, engine, mixed_switch_rtol)
    _lib.check(_LIB.cdft_batch_converge(plans, n, ptrs, ctypes.byref(opts), res))
    return [ConvergeResult(res[i], None) for i in range(n)]


def dFdrho_res(system, rho):
    """δFδρ_res(system, ρ) (models.jl:194-200): residual functional derivative
    plus external field, in k_B T, shape (nc, N)."""
    _check_rho(system, rho)
    out = np.empty_like(rho)
    _lib.check(_LIB.cdft_functional_derivative(system._plan, _lib.dptr(rho), _lib.dptr(out)))
    return out


def bulk_density(model, p, T, x=None, phase="stable"):
    """Molar densities (mol/m^3) at pressures ``p`` (scalar or array, Pa), temperature T and
    mole fractions ``x`` (one composition, or one row per pressure), solved on the device in
    one launch (cdft_bulk_density): "stable" (the lower-Gibbs-energy root, as
    PCSAFT.stable_density and Clapeyron's volume(model, p, T, x)), "liquid" (densest root)
    or "vapour" (most dilute).  Models with cross-association are refused (use
    PCSAFT.stable_density)."""
    p = np.atleast_1d(np.asarray(p, dtype=np.float64))
    n = p.size
    nc = len(model)
    x = np.ones(nc) if x is None else np.asarray(x, dtype=np.float64)
    x = np.ascontiguousarray(np.broadcast_to(x.reshape(-1, nc), (n, nc)))
    d = _lib.SystemDesc()
    d.nc = nc
    size = model.d(T)
    for i in range(nc):
        d.m[i] = model.m[i]
        d.hsd[i] = size[i]
        for j in range(nc):
            d.sigma[i * nc + j] = model.sigma_ij[i, j]
            d.eps[i * nc + j] = model.eps_ij[i, j]
    d.L = model.length_scale()
    d.T = T
    pairs = model.assoc_pairs()
    d.n_assoc = len(pairs)
    for q, (i, a, j, b, eab, kab) in enumerate(pairs):
        d.assoc[q] = _lib.AssocPair(i, j, a, b, 1, 1, eab, kab)
    rho = np.empty(n)
    status = np.zeros(n, dtype=np.int32)
    code = {"stable": 0, "liquid": 1, "vapour": 2}[phase]
    _lib.check(_LIB.cdft_bulk_density(ctypes.byref(d), n, _lib.dptr(p), _lib.dptr(x), code, _lib.dptr(rho),
                                      status.ctypes.data_as(ctypes.c_void_p)))
    if np.any(status != 0):
        raise ValueError(f"no density root at pressures {p[status != 0]}")
    return rho


def saturation(model, T):
    """Pure-component vapour-liquid coexistence at temperatures ``T`` (scalar or array, K),
    solved on the device in one launch (cdft_saturation_pure): arrays (p_sat [Pa],
    rho_liquid, rho_vapour [mol/m^3]).  The saturation state that surface_tension(model, T, x)
    takes from bubble_pressure for a pure component (surface_tension.jl:13-20); the host
    equivalent is PCSAFT.saturation."""
    if len(model) != 1:
        raise ValueError("saturation of a pure component")
    T = np.atleast_1d(np.asarray(T, dtype=np.float64))
    n = T.size
    d = _lib.SystemDesc()
    d.nc = 1
    d.m[0] = model.m[0]
    d.hsd[0] = model.d(float(T[0]))[0]
    d.sigma[0] = model.sigma_ij[0, 0]
    d.eps[0] = model.eps_ij[0, 0]
    d.L = model.length_scale()
    d.T = float(T[0])
    pairs = model.assoc_pairs()
    d.n_assoc = len(pairs)
    for q, (i, a, j, b, eab, kab) in enumerate(pairs):
        d.assoc[q] = _lib.AssocPair(i, j, a, b, 1, 1, eab, kab)
    p, rl, rv = np.empty(n), np.empty(n), np.empty(n)
    status = np.zeros(n, dtype=np.int32)
    _lib.check(_LIB.cdft_saturation_pure(ctypes.byref(d), n, _lib.dptr(T), _lib.dptr(p), _lib.dptr(rl),
                                         _lib.dptr(rv), status.ctypes.data_as(ctypes.c_void_p)))
    if np.any(status != 0):
        raise ValueError(f"no coexistence at T = {T[status != 0]} (status {status[status != 0]})")
    return p, rl, rv


def ddft_rhs(system, eta):
    """The right-hand side of dynamic DFT in eta = ln rho, the function ddft_rhs_log! that
    SciMLBase.ODEProblem(system, ρ, tspan) integrates (ext/SciMLBasecDFTExt.jl:10-61):
    lap(eta) + lap(mu) + grad eta . (grad eta + grad mu), mu = dF/drho_res + V_ext, rho =
    exp(clamp(eta, -50, 30)), spectral derivatives in reduced lengths; shape (nc, grid...)."""
    eta = np.ascontiguousarray(eta, dtype=np.float64)
    _check_rho(system, eta)
    out = np.empty_like(eta)
    _lib.check(_LIB.cdft_ddft_rhs(system._plan, _lib.dptr(eta), _lib.dptr(out)))
    return out


def ddft_problem(system, rho, tspan):
    """SciMLBase.ODEProblem(system, ρ, tspan) (ext/SciMLBasecDFTExt.jl:10-61) as the triple
    (f, u0, tspan): f(u, t) -> du/dt with u = ln rho, u0 = log(rho); any ODE integrator
    (scipy.integrate.solve_ivp on the raveled state, say) takes it from here."""
    shape = np.shape(rho)

    def f(u, t=None):
        return ddft_rhs(system, np.reshape(u, shape)).reshape(np.shape(u))

    return f, np.log(np.asarray(rho, dtype=np.float64)), tuple(tspan)


def phi_pointwise(system, n):
    """Fused Phi and dPhi/dn at points; n has shape (nc, NF, npts)."""
    n = np.ascontiguousarray(n, dtype=np.float64)
    npts = n.shape[-1]
    f = np.empty(npts)
    g = np.empty_like(n)
    _lib.check(_LIB.cdft_phi_pointwise(system._plan, _lib.dptr(n), npts, _lib.dptr(f), _lib.dptr(g)))
    return f, g


class _KSum:
    def __init__(self):
        self.s = 0.0
        self.c = 0.0

    def add(self, x):
        t = self.s + x
        if abs(self.s) >= abs(x):
            self.c += (self.s - t) + x
        else:
            self.c += (x - t) + self.s
        self.s = t

    def value(self):
        return self.s + self.c


def integrate(f, structure):
    """``∫(f, structure)`` (integrals.jl:17,28-41): Simpson weights 1,4,2,...,1 per
    dimension (outer product), dz = (ub-lb)/N, compensated FP64 summation."""
    f = np.asarray(f, dtype=float)
    if getattr(structure, "coord", "cart") != "cart":   # 4 pi / 2 pi integrateR (integrals.jl:18-19)
        acc = _KSum()
        for v in (structure.weights * f).ravel():
            acc.add(float(v))
        return acc.value()
    w = np.ones(())
    for ax, n in enumerate(f.shape):
        k = np.arange(1, n + 1)
        c = np.where((k == 1) | (k == n), 1.0, np.where(k % 2 == 0, 4.0, 2.0))
        shape = [1] * f.ndim
        shape[ax] = n
        w = w * c.reshape(shape)
    terms = (w * f).ravel()
    if terms.size > 100000:          # large 3D grids: pairwise (NumPy) summation
        total = float(np.sum(terms))
    else:
        acc = _KSum()
        for v in terms:
            acc.add(float(v))
        total = acc.value()
    return total * float(np.prod(np.array(structure.dz()) / 3))


def F_res(system, rho):
    """F_res(system, ρ) (models.jl:86-91), per unit area, in k_B T."""
    _check_rho(system, rho)
    out = ctypes.c_double()
    _lib.check(_LIB.cdft_free_energy_res(system._plan, _lib.dptr(rho), ctypes.byref(out)))
    return out.value


def batch_integrals(systems, rhos=None):
    """The integrals of several systems on the device in one batch (cdft_batch_integrals):
    per system a dict with F_res and F_ideal (k_B T), int_rho (per component) and int_one.
    ``rhos`` None takes the profiles the plans hold (right after a converge)."""
    n = len(systems)
    nc = systems[0].nc
    nq = 3 + nc
    out = np.zeros(n * nq)
    plans = (ctypes.c_void_p * n)(*[s._plan.value for s in systems])
    if rhos is None:
        ptrs = None
    else:
        for s, r in zip(systems, rhos):
            _check_rho(s, r)
        ptrs = (ctypes.c_void_p * n)(*[r.ctypes.data for r in rhos])
    _lib.check(_LIB.cdft_batch_integrals(plans, n, ptrs, 0, _lib.dptr(out)))
    res = []
    for k in range(n):
        q = out[k * nq:(k + 1) * nq]
        res.append({"F_res": float(q[0]), "F_ideal": float(q[1]), "int_rho": q[2:2 + nc].copy(),
                    "int_one": float(q[2 + nc])})
    return res


def _integrals(system, rho):
    return batch_integrals([system], [rho])[0]


def F_ideal(system, rho):
    """F_ideal(system, ρ) (BasicIdeal.jl:10-38), on the device."""
    return _integrals(system, rho)["F_ideal"]


def free_energy(system, rho):
    """free_energy(system, ρ) = F_ideal + F_res (src/utils/base.jl:8-10), on the device."""
    q = _integrals(system, rho)
    return q["F_ideal"] + q["F_res"]


def _omega_ex(system, q):
    s = system.structure
    p, T = s.conditions
    mu = system.model.chemical_potential(s.rho_bulk, T)
    F = q["F_ideal"] + q["F_res"]
    return F * K_B * T - float(np.dot(mu, q["int_rho"])) + p * q["int_one"]


def surface_tension(system, rho, x=None):
    """surface_tension(system, ρ) (surface_tension.jl:31-53), J/m^2; the
    periodic two-interface seed gives twice the tension (callers divide by 2).
    The integrals run on the device (cdft_batch_integrals).

    surface_tension(model, T, x=[1.0]) (surface_tension.jl:13-29), for a pure component and
    one or many temperatures T: the coexistence of every T from one device launch
    (cdft_saturation_pure, the state bubble_pressure gives the reference), a TwoPhase1DCart
    on [-10L, 10L] with 201 points per T, the systems converged together (converge!'s
    default solver) and surface_tension(system, ρ) / 2.  Returns gamma (J/m^2), a float for
    a scalar T, else an array."""
    if isinstance(system, PCSAFT):
        return _surface_tension_model(system, rho, x)
    return _omega_ex(system, _integrals(system, rho))


def _surface_tension_model(model, T, x=None):
    if x is not None and (len(x) != 1 or float(x[0]) != 1.0):
        raise ValueError("surface_tension(model, T, x) covers pure components (x = [1.0])")
    scalar = np.ndim(T) == 0
    Ts = np.atleast_1d(np.asarray(T, dtype=np.float64))
    p, rl, rv = saturation(model, Ts)
    L = model.length_scale()
    systems = [DFTSystem(model, TwoPhase1DCart((float(pk), float(Tk)), [float(lk)], [float(vk)], [-10 * L, 10 * L], 201))
               for pk, Tk, lk, vk in zip(p, Ts, rl, rv)]
    rhos = [initialize_profiles(sy) for sy in systems]
    batch_converge(systems, rhos)
    gam = np.array([surface_tension(sy, r) / 2 for sy, r in zip(systems, rhos)])
    for sy in systems:
        sy.close()
    return float(gam[0]) if scalar else gam


def interfacial_tension(system, rho):
    """interfacial_tension(system, ρ) == surface_tension(system, ρ) (interfacial_tension.jl:63)."""
    return surface_tension(system, rho)


def _domain_volume(st):
    return st.volume() if hasattr(st, "volume") else float(np.prod([ub - lb for (lb, ub) in st.bounds]))


def adsorption(system, rho):
    """adsorption(system, ρ) (adsorption.jl:26-32), mol/m^3 of the domain."""
    return _integrals(system, rho)["int_rho"] / _domain_volume(system.structure)


def batch_properties(systems, rhos=None):
    """Excess grand potential (surface_tension's numerator, J/m^2 in 1D) and adsorption of
    several systems from one batched device call."""
    out = []
    for sy, q in zip(systems, batch_integrals(systems, rhos)):
        out.append({"omega_ex": _omega_ex(sy, q), "adsorption": q["int_rho"] / _domain_volume(sy.structure),
                    "free_energy": q["F_ideal"] + q["F_res"]})
    return out


def F_res_grad(system, rho):
    """dF_res/d(sigma_k [A], eps_k/k_B [K], m_k) at a fixed profile, shape (nc, 3);
    units of F_res (k_B T per m^2 in 1D, k_B T in 3D).  No counterpart in the reference."""
    _check_rho(system, rho)
    out = np.zeros(3 * system.nc)
    _lib.check(_LIB.cdft_free_energy_res_grad(system._plan, _lib.dptr(rho), _lib.dptr(out)))
    return out.reshape(system.nc, 3)


def grad_params(system, rho, dmu_dtheta=None, dp_dtheta=None):
    """d Omega / d(sigma_k [A], eps_k/k_B [K], m_k) at a converged profile, shape (nc, 3),
    J/m^2 per parameter unit.  Without an external field Omega is surface_tension's
    numerator; with planar Steele walls it is the grand potential including the wall term
    (grand_potential), the functional converge! makes stationary.  dmu_dtheta (nc, 3nc) and
    dp_dtheta (3nc) describe how the bulk state moves with the parameters (None: held fixed)."""
    _check_rho(system, rho)
    nt = 3 * system.nc
    out = np.zeros(nt)
    mu = None if dmu_dtheta is None else np.ascontiguousarray(dmu_dtheta, dtype=float).reshape(system.nc, nt)
    dp = None if dp_dtheta is None else np.ascontiguousarray(dp_dtheta, dtype=float).reshape(nt)
    mu_p = None if mu is None else _lib.dptr(mu)
    dp_p = None if dp is None else _lib.dptr(dp)
    if system.vext is None:
        _lib.check(_LIB.cdft_grad_params(system._plan, _lib.dptr(rho), mu_p, dp_p, _lib.dptr(out)))
    else:
        st = system.structure
        T = st.conditions[1]
        if st.coord == "cart" and st.nd == 3 and all(isinstance(f, HardSphereSolutes) for f in system.external_field):
            # V_ext / k_B T of hard solutes is a constant height: no parameter dependence
            dv = np.zeros((nt, system.nc) + tuple(reversed(st.ngrid)))
        elif st.nd == 1 and st.coord == "cart" and all(isinstance(f, Steele) for f in system.external_field):
            z = st.coords(0)
            dv = np.ascontiguousarray(sum(f.potential_dtheta(system.model, z, T) for f in system.external_field))
        else:
            raise NotImplementedError("parameter gradients with external fields: planar Steele walls, hard solutes")
        _lib.check(_LIB.cdft_grad_params_ext(system._plan, _lib.dptr(rho), mu_p, dp_p, _lib.dptr(dv), _lib.dptr(out)))
    return out.reshape(system.nc, 3)


def grand_potential(system, rho, quadrature="simpson"):
    """The grand potential per unit area (1D) that converge! makes stationary, J/m^2:
    F k_B T + R T sum_i int rho_i V_i - sum_i mu_i int rho_i + p int 1 (surface_tension's
    numerator plus the external-field energy; rho in mol/m^3, V in k_B T).
    quadrature "simpson": the weights of surface_tension (integrals.jl:28-41); "uniform":
    the weights dz of the discrete functional whose gradient the pointwise Euler-Lagrange
    equation is -- the converged profile is its exact stationary point, and grad_params is
    its exact parameter derivative."""
    T = system.structure.conditions[1]
    if quadrature == "simpson":
        om = surface_tension(system, rho)
        if system.vext is None:
            return om
        return om + N_A * K_B * T * sum(integrate(rho[i] * system.vext[i], system.structure)
                                        for i in range(system.nc))
    if quadrature != "uniform":
        raise ValueError("quadrature is 'simpson' or 'uniform'")
    st = system.structure
    if st.coord != "cart":
        raise NotImplementedError("the uniform quadrature is defined for Cartesian grids")
    dv = float(np.prod([(ub - lb) / n for (lb, ub), n in zip(st.bounds, st.ngrid)]))   # volume per point
    n_pts = int(np.prod(st.ngrid))
    p, _ = st.conditions
    mu = system.model.chemical_potential(st.rho_bulk, T)
    f_res = _uniform_F_res(system, rho)
    f_id = sum(float(np.sum(N_A * rho[i] * (np.log(rho[i]) - 1.5 * np.log(T) - 1))) for i in range(system.nc)) * dv
    om = (f_res + f_id) * K_B * T - sum(mu[i] * float(np.sum(rho[i])) * dv for i in range(system.nc)) + p * n_pts * dv
    if system.vext is not None:
        om += N_A * K_B * T * sum(float(np.sum(rho[i] * system.vext[i])) for i in range(system.nc)) * dv
    return om


def _uniform_F_res(system, rho):
    """F_res (k_B T per m^2 in 1D, k_B T in 3D) summed with uniform weights: Phi at every point
    from the device (cdft_phi_field)."""
    _check_rho(system, rho)
    st = system.structure
    f = np.empty(int(np.prod(st.ngrid)))
    _lib.check(_LIB.cdft_phi_field(system._plan, _lib.dptr(rho), _lib.dptr(f)))
    dv = float(np.prod([(ub - lb) / n for (lb, ub), n in zip(st.bounds, st.ngrid)]))
    return float(np.sum(f)) * dv / system.L ** 3


def dgamma_dtheta(system, rho):
    """d gamma / d(sigma_k [A], eps_k/k_B [K], m_k) of a converged TwoPhase1DCart
    interface (periodic box, two interfaces: gamma = Omega_ex / 2), shape (nc, 3),
    J/m^2 per parameter unit.  The bulk state follows phase coexistence (pure fluid:
    saturation; binary: fixed p and T); its sensitivity comes from
    thermo.coexistence_sensitivity."""
    s = system.structure
    if s.kind != "twophase":
        raise ValueError("dgamma_dtheta needs a TwoPhase1DCart structure")
    p, T = s.conditions
    from .thermo import coexistence_sensitivity
    dmu, dp = coexistence_sensitivity(system.model, T, s.rho_bulk, s.rho_bulk2, p=p)
    return grad_params(system, rho, dmu, dp) / 2


def tuning(name, value=None):
    """Get (and with ``value``, first set) a launch shape of the autotuner by name,
    process-wide (cdft_tuning_get / cdft_tuning_set)."""
    if value is not None:
        _lib.check(_LIB.cdft_tuning_set(name.encode(), int(value)))
    out = ctypes.c_int()
    _lib.check(_LIB.cdft_tuning_get(name.encode(), ctypes.byref(out)))
    return out.value


def launch_count(reset=False):
    return _LIB.cdft_launch_count(1 if reset else 0)
