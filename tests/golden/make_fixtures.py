"""Generate the oracle fixtures of the benchmark configurations at their own sizes.

Test infrastructure: runs the CPU oracle (``oracle/``, a NumPy restatement of the
reference's converge! path) on the five benchmark configurations and writes
compressed ``.npz`` files next to this script.  The ``-m gpu`` tests
(``tests/test_gpu_configs.py``) build the same systems from the stored inputs and
compare the CUDA path with these outputs.

    python tests/golden/make_fixtures.py [--only c1,c2,c3,c4,c5,a9] [--jobs 8]

Configurations (synthetic state points, explicit PC-SAFT parameters):

* c1 -- methane liquid (150 K, 10 MPa) next to one graphite Steele wall,
  201 points on [0.5 sigma, 4.5 sigma]; beta 0.1, m 5, tol 1e-13.
* c2 -- n-octane vapour-liquid interface at 298.15 K, 2048 points over 40 sigma
  (TwoPhase1DCart, two interfaces); beta 0.01 (the converge! default), m 5, tol 1e-13.
* c3 -- the 64-point slit-pore isotherm: methane at 150 K in graphite slits of
  8 widths 2-8 nm x 8 pressures 1e3-1e7 Pa, N = 100..400 linear in the width,
  bounds [0.7 sigma, H - 0.7 sigma] as adsorption(model, surface, p, T) builds them
  (src/methods/adsorption.jl:48-65); beta 0.1, m 5, tol 1e-13.
* c4 -- water (2B association) + n-octane liquid-liquid interface, 298.15 K,
  1e5 Pa, 4096 points over 60 sigma_water; beta 0.01, m 5, tol 1e-12 (converged by the
  oracle's C++ restatement, oracle/cpu_converge.cpp, which agrees with the NumPy oracle
  to 1e-11 in dF/drho; the NumPy run takes hours at this size).
* c5 -- argon at 100 K, rho_b = 0.021 A^-3, periodic 128^3 box of edge 16 sigma with
  27 hard spherical solutes (radius 1.5 sigma, numpy default_rng(0)); beta 0.1,
  m 10, tol 1e-11 (the FFT path's FP64 residual floor on this box sits near
  1e-12 ||r0||).  The converged profile is stored on every 4th point per axis.

* a9 -- water + ethanol liquid (x = 0.5/0.5, 298.15 K, 1e5 Pa) next to one graphite
  Steele wall, 150 points on [0.5 sigma_water, 4.5 sigma_water]: self- and
  cross-association, 4 site pairs, the general association solve (assoc.jl:771-828);
  beta 0.01, m 5, tol 1e-12.  Not one of the five benchmark configurations: the parity
  case of the general association path.

Every configuration is converged twice: with the oracle's default White-Bear
bracket (a 16-term Taylor series for |n3| < 0.05, elsewhere the reference's closed
form, FMT.jl:39-45) and with the reference's literal closed form everywhere; the
fixture records how far the two fixed points are apart.
"""
import argparse
import multiprocessing as mp
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

PARAMS = {
    "methane": (1.0, 3.7039, 150.03),
    "octane": (3.8176, 3.8373, 242.78),
    "water": (1.0656, 3.0007, 366.51),
    "argon": (1.0, 3.4, 120.0),
    "ethanol": (2.3827, 3.1771, 198.24),
}
WATER_ASSOC = (2500.7, 0.034868)
ASSOC = {"water": WATER_ASSOC, "ethanol": (2653.4, 0.032384)}

ISO_T = 150.0
ISO_WIDTHS = np.linspace(2e-9, 8e-9, 8)
ISO_PRESSURES = np.logspace(3, 7, 8)
ISO_N = [int(round(100 + 300 * k / 7)) for k in range(8)]


def oracle_model(names):
    from oracle import pcsaft_bulk as pb
    m = [PARAMS[n][0] for n in names]
    s = [PARAMS[n][1] for n in names]
    e = [PARAMS[n][2] for n in names]
    assoc = [(i, i, ASSOC[n][0], ASSOC[n][1]) for i, n in enumerate(names) if n in ASSOC]
    # cross-association between two associating components by the Elliott rule
    for i, a in enumerate(names):
        for j, b in enumerate(names):
            if j > i and a in ASSOC and b in ASSOC:
                sij = 0.5 * (s[i] + s[j])
                k = np.sqrt(ASSOC[a][1] * ASSOC[b][1]) * (np.sqrt(s[i] * s[j]) / sij) ** 3
                assoc.append((i, j, 0.5 * (ASSOC[a][0] + ASSOC[b][0]), float(k)))
    return pb.PCSAFTModel(list(names), m, s, e, assoc=assoc)


def isotherm_specs():
    """(width m, pressure Pa, N) of the 64 state points, widths outer, pressures inner."""
    return [(float(H), float(p), ISO_N[k]) for k, H in enumerate(ISO_WIDTHS) for p in ISO_PRESSURES]


def stable_bulk_density(om, p, T):
    """The bulk density of the stable phase at (p, T) (the root of lower Gibbs energy)."""
    from oracle import pcsaft_bulk as pb
    roots = []
    for ph in ("liquid", "vapour"):
        try:
            roots.append(pb.density(om, p, T, [1.0], ph))
        except RuntimeError:
            pass
    if len(roots) == 2 and abs(roots[0] / roots[1] - 1) > 1e-10:
        g = [pb.mu_total(om, [r], T)[0] for r in roots]
        return roots[0] if g[0] <= g[1] else roots[1]
    return roots[0]


def _converge(so, kw, closed=False):
    so.wb_closed = closed
    rho0 = so.initialize_profiles()
    t = time.perf_counter()
    with np.errstate(all="ignore"):
        rho, out = so.converge(rho0, **kw)
    return rho, out, time.perf_counter() - t


class _CppOut:
    def __init__(self, res):
        self.errcode = res.errcode
        self.history = np.zeros(res.evaluations)


def _converge_cpp(so, kw, closed=False):
    """The same converge! through the oracle's C++ restatement (oracle/cpu_converge.cpp),
    for the 1D configurations whose NumPy runs take too long (4096 points, two components)."""
    from oracle import cpu
    cpu.build()
    cpu.set_wb_closed(closed)
    rho = [np.ascontiguousarray(so.initialize_profiles())]
    t = time.perf_counter()
    res, _ = cpu.batch_converge([so], rho, nthreads=1, **kw)
    cpu.set_wb_closed(False)
    return rho[0], _CppOut(res[0]), time.perf_counter() - t


def _excess_omega(so, rho):
    with np.errstate(all="ignore"):
        return float(so.surface_tension(rho))


# ---------------------------------------------------------------------------
def case_c1():
    from oracle import functional as fn, pcsaft_bulk as pb
    om = oracle_model(["methane"])
    T, p, N = 150.0, 1e7, 201
    rb = pb.density(om, p, T, [1.0])
    s = om.sigma[0]
    bounds = (0.5 * s, 4.5 * s)
    so = fn.DFTSystem(om, fn.Structure((p, T), [rb], [bounds], (N,)), [fn.SteeleWall.graphite()])
    kw = dict(beta=0.1, tol=1e-13, anderson_m=5, maxit=10000)
    rho, out, dt = _converge(so, kw)
    rc, outc, _ = _converge(so, kw, closed=True)
    return "c1_methane_wall_201", dict(
        T=T, p=p, N=N, rho_bulk=[rb], bounds=bounds, rho=rho, errcode=out.errcode, evaluations=len(out.history),
        F_res=so.F_res(rho), omega_ex=_excess_omega(so, rho), adsorption=so.adsorption(rho),
        closed_errcode=outc.errcode, closed_rho_rel_diff=float(np.max(np.abs(rc / rho - 1))),
        closed_omega_rel_diff=abs(_excess_omega(so, rc) / _excess_omega(so, rho) - 1), seconds=dt)


def case_c2():
    from oracle import functional as fn, pcsaft_bulk as pb
    om = oracle_model(["octane"])
    T, N = 298.15, 2048
    psat, rl, rv = pb.saturation_pure(om, T)
    s = om.sigma[0]
    bounds = (-20 * s, 20 * s)
    so = fn.DFTSystem(om, fn.Structure((psat, T), [rl], [bounds], (N,), kind="twophase", rho_bulk2=[rv]))
    kw = dict(beta=0.01, tol=1e-13, anderson_m=5, maxit=20000)
    rho, out, dt = _converge(so, kw)
    rc, outc, _ = _converge(so, kw, closed=True)
    g = _excess_omega(so, rho) / 2
    gc = _excess_omega(so, rc) / 2
    return "c2_octane_vle_2048", dict(
        T=T, p=psat, N=N, rho_bulk=[rl], rho_bulk2=[rv], bounds=bounds, rho=rho, errcode=out.errcode,
        evaluations=len(out.history), gamma=g, closed_errcode=outc.errcode,
        closed_rho_rel_diff=float(np.max(np.abs(rc / rho - 1))), closed_gamma_rel_diff=abs(gc / g - 1), seconds=dt)


def case_c3_point(k):
    """One isotherm state point (index k of isotherm_specs())."""
    from oracle import functional as fn
    H, p, N = isotherm_specs()[k]
    om = oracle_model(["methane"])
    rb = stable_bulk_density(om, p, ISO_T)
    s = om.sigma[0]
    so = fn.DFTSystem(om, fn.Structure((p, ISO_T), [rb], [(0.7 * s, H - 0.7 * s)], (N,)), [fn.SteeleWall.graphite(H)])
    kw = dict(beta=0.1, tol=1e-13, anderson_m=5, maxit=10000)
    rho, out, dt = _converge(so, kw)
    rc, outc, _ = _converge(so, kw, closed=True)
    om_s, om_c = _excess_omega(so, rho), _excess_omega(so, rc)
    ad_s, ad_c = so.adsorption(rho)[0], so.adsorption(rc)[0]
    return dict(k=k, H=H, p=p, N=N, rho_bulk=rb, rho=rho[0], errcode=out.errcode, evaluations=len(out.history),
                adsorption=ad_s, omega_ex=om_s, closed_errcode=outc.errcode,
                closed_rho_rel_diff=float(np.max(np.abs(rc / rho - 1))),
                closed_omega_rel_diff=abs(om_c / om_s - 1), closed_adsorption_rel_diff=abs(ad_c / ad_s - 1),
                seconds=dt)


def collect_c3(points):
    points = sorted(points, key=lambda d: d["k"])
    offs = np.cumsum([0] + [d["N"] for d in points])
    out = {key: np.array([d[key] for d in points]) for key in points[0] if key != "rho"}
    out["rho"] = np.concatenate([d["rho"] for d in points])
    out["offsets"] = offs
    out["T"] = ISO_T
    return "c3_isotherm64", out


def case_c4():
    from oracle import functional as fn, pcsaft_bulk as pb
    om = oracle_model(["water", "octane"])
    T, p, N = 298.15, 1e5, 4096
    x1, x2 = pb.lle_binary(om, p, T)
    r1 = pb.density(om, p, T, x1) * x1
    r2 = pb.density(om, p, T, x2) * x2
    s = om.sigma[0]
    bounds = (-30 * s, 30 * s)
    so = fn.DFTSystem(om, fn.Structure((p, T), list(r1), [bounds], (N,), kind="twophase", rho_bulk2=list(r2)))
    kw = dict(beta=0.01, tol=1e-12, anderson_m=5, maxit=40000)
    rho, out, dt = _converge_cpp(so, kw)
    rc, outc, _ = _converge_cpp(so, kw, closed=True)
    g = _excess_omega(so, rho) / 2
    gc = _excess_omega(so, rc) / 2
    return "c4_water_octane_lle_4096", dict(
        T=T, p=p, N=N, x1=x1, x2=x2, rho_bulk=r1, rho_bulk2=r2, bounds=bounds, rho=rho, errcode=out.errcode,
        evaluations=len(out.history), gamma=g, closed_errcode=outc.errcode,
        closed_rho_rel_diff=float(np.max(np.abs(rc / rho - 1))), closed_gamma_rel_diff=abs(gc / g - 1), seconds=dt)


def case_a9():
    from oracle import functional as fn, pcsaft_bulk as pb
    om = oracle_model(["water", "ethanol"])
    p, T = 1e5, 298.15
    x = np.array([0.5, 0.5])
    rb = x * pb.density(om, p, T, x, "liquid")
    s = om.sigma[0]
    so = fn.DFTSystem(om, fn.Structure((p, T), rb, [(0.5 * s, 4.5 * s)], (150,)), [fn.SteeleWall.graphite(0.0)])
    kw = dict(beta=0.01, tol=1e-12, anderson_m=5, maxit=10000)
    rho, out, dt = _converge(so, kw)
    rc, outc, _ = _converge(so, kw, closed=True)
    return "a9_water_ethanol_wall_150", dict(
        p=p, T=T, x=x, rho_bulk=rb, N=150, rho=rho, errcode=out.errcode, evaluations=len(out.history),
        adsorption=so.adsorption(rho), omega_ex=_excess_omega(so, rho),
        closed_errcode=outc.errcode, closed_rho_rel_diff=float(np.max(np.abs(rc / rho - 1))), seconds=dt)


def solute_centres(n, radius, box, min_gap, seed=0):
    """n non-overlapping centres in [0, box)^3 by rejection sampling with
    numpy.random.default_rng(seed); minimum-image centre distances >= 2 radius + min_gap."""
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


def solute_vext(N, box, centres, radius, height=100.0):
    """V_ext / k_B T of hard spherical solutes on the periodic N^3 grid LinRange(0, box, N)."""
    x = np.linspace(0.0, box, N)
    X, Y, Z = x[None, None, :], x[None, :, None], x[:, None, None]
    inside = np.zeros((N, N, N), dtype=bool)
    for c in centres:
        dx = X - c[0]
        dx = dx - box * np.round(dx / box)
        dy = Y - c[1]
        dy = dy - box * np.round(dy / box)
        dz = Z - c[2]
        dz = dz - box * np.round(dz / box)
        inside |= dx * dx + dy * dy + dz * dz < radius ** 2
    return np.where(inside, height, 0.0)[None]


def case_c5(N=128, stride=4):
    from oracle import functional as fn, pcsaft_bulk as pb
    om = oracle_model(["argon"])
    T = 100.0
    s = om.sigma[0]
    box = 16.0 * s
    rb = 0.021e30 / pb.N_A
    centres = solute_centres(27, 1.5 * s, box, 2 * box / N, seed=0)
    V = solute_vext(N, box, centres, 1.5 * s)
    so = fn.DFTSystem(om, fn.Structure((1e5, T), [rb], [(0.0, box)] * 3, (N, N, N)), vext=V)
    kw = dict(beta=0.1, tol=1e-11, anderson_m=10, maxit=1000)
    rho, out, dt = _converge(so, kw)
    fluid = V[0] == 0
    # the closed bracket loses every digit where n3 crosses zero next to the solutes; its run
    # is capped at 40 evaluations and compared where it stopped
    kwc = dict(kw, maxit=40)
    rc, outc, _ = _converge(so, kwc, closed=True)
    om_s = _excess_omega(so, rho)
    om_c = _excess_omega(so, rc)
    sub = (slice(None), slice(None, None, stride), slice(None, None, stride), slice(None, None, stride))
    return "c5_solutes_128", dict(
        T=T, p=1e5, N=N, rho_bulk=[rb], box=box, centres=centres, radius=1.5 * s, stride=stride,
        rho_sub=rho[sub], fluid_sum=float(np.sum(rho[0][fluid])), fluid_sumsq=float(np.sum(rho[0][fluid] ** 2)),
        errcode=out.errcode, evaluations=len(out.history), omega_ex=om_s, F=float(so.free_energy(rho)),
        closed_errcode=outc.errcode, closed_evaluations=len(outc.history),
        closed_resnorm_ratio=float(outc.history[-1] / outc.history[0]),
        closed_rho_rel_diff_fluid=float(np.max(np.abs(rc[0][fluid] / rho[0][fluid] - 1))),
        closed_omega_rel_diff=abs(om_c / om_s - 1), seconds=dt)


def _run(task):
    name, arg = task
    t = time.perf_counter()
    if name == "c3":
        res = case_c3_point(arg)
    else:
        res = {"c1": case_c1, "c2": case_c2, "c4": case_c4, "c5": case_c5, "a9": case_a9}[name]()
    print(f"{name}{'' if arg is None else arg} done in {time.perf_counter() - t:.1f} s", flush=True)
    return name, res


def save(name, data):
    path = os.path.join(HERE, name + ".npz")
    np.savez_compressed(path, **{k: np.asarray(v) for k, v in data.items()})
    print("wrote", os.path.relpath(path, ROOT), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--only", default="c1,c2,c3,c4,c5,a9")
    ap.add_argument("--jobs", type=int, default=os.cpu_count() or 1)
    args = ap.parse_args()
    want = args.only.split(",")
    # the long single cases first, then the 64 isotherm points fill the other workers
    tasks = [(c, None) for c in ("c5", "c4", "c2", "c1", "a9") if c in want]
    if "c3" in want:
        tasks += [("c3", k) for k in range(len(isotherm_specs()))]
    c3 = []
    with mp.get_context("spawn").Pool(args.jobs) as pool:
        for name, res in pool.imap_unordered(_run, tasks):
            if name == "c3":
                c3.append(res)
            else:
                save(*res)
    if c3:
        save(*collect_c3(c3))


if __name__ == "__main__":
    main()
