"""Autotuner of the library's launch shapes (the entries of csrc/tuning.cuh).

Every entry is swept on the workload it governs, timed with CUDA events after warm-up,
and the fastest value is reported with the time of every candidate:

* pers_warp_aa_max_elem -- persistent engine, Anderson section on one warp for systems of
  at most this many elements: the 64-point slit-pore isotherm (N = 100..400), batched; the
  objective is the time per evaluation of the critical path (batch time over the largest
  evaluation count), because a few state points' evaluation counts are chaotic in the last
  bits of their arithmetic.
* fft3d_tma, fft3d_fused_phi -- 3D grids: TMA tile kernels for the y/z passes, the fused
  x pass with Phi: one functional derivative of the 27-solute argon box at 64^3 and
  128^3, FP64 and mixed.
* radial_dmma -- radial grids: the batch's dense operators as tensor-core GEMMs over column
  tiles of state points sharing an operator, or per-system warp-per-row launches: the dense
  stage of the 64-point spherical-pore isotherm (one launch for the batch).

    python cdft.jl_b200/tune.py [--out tuning.json]

The entries that change arithmetic (the warp Anderson section reduces in another order)
are per-system rules, so a sweep can set them freely; the defaults compiled into the
library are the winners of this sweep on B200.
"""
import argparse
import ctypes
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
for p in (HERE, ROOT):
    if p not in sys.path:
        sys.path.insert(0, p)


def _events(fn, reps, warm=2):
    import torch
    for _ in range(warm):
        fn()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        fn()
    e1.record()
    e1.synchronize()
    return e0.elapsed_time(e1) / reps


def sweep_isotherm(values=(0, 256, 512, 1024)):
    """ms per batch, the largest evaluation count, and their ratio (the time per evaluation
    of the critical path: the objective, since a few state points' evaluation counts are
    chaotic in the last bits and the entry changes summation orders)."""
    import cdft_b200 as cd
    import bench
    systems, rho0 = bench.build_systems(bench.isotherm_specs(0), "fp64")
    method = cd.AASol.for_system(None, **bench.SOLVER)
    out = {}
    for v in values:
        cd.tuning("pers_warp_aa_max_elem", v)
        evals = []

        def run():
            rr = [r.copy() for r in rho0]
            res = cd.batch_converge(systems, rr, method=method)
            evals[:] = [r.evaluations for r in res]

        ms = _events(run, 3)
        out[v] = {"ms_per_batch": ms, "max_evaluations": max(evals), "us_per_critical_evaluation": 1e3 * ms / max(evals)}
    return out


def sweep_3d(sizes=(64, 128), precisions=("fp64", "mixed")):
    import cdft_b200 as cd
    import bench
    from cdft_b200 import _lib
    lib = _lib.load()
    out = {}
    for N in sizes:
        for prec in precisions:
            sy = bench._solutes3d_system(N, prec)
            rho = cd.initialize_profiles(sy)
            plans = (ctypes.c_void_p * 1)(sy._plan.value)
            cd.dFdrho_res(sy, rho)   # the plan's device profile
            for tma, fused in ((0, 0), (1, 0), (1, 1)):
                cd.tuning("fft3d_tma", tma)
                cd.tuning("fft3d_fused_phi", fused)
                ms = ctypes.c_double()
                _lib.check(lib.cdft_batch_time_stage(plans, 1, 3, 20, ctypes.byref(ms)))
                out[f"{N}^3 {prec} tma={tma} fused={fused}"] = ms.value
            sy.close()
    return out


def sweep_radial():
    """ms per dense stage of the spherical-pore isotherm batch, per radial_dmma value."""
    import cdft_b200 as cd
    import bench
    from cdft_b200 import _lib
    lib = _lib.load()
    model = cd.PCSAFT(["methane"], **bench.METHANE)
    specs = [(float(R), float(p), bench.N_OF_RADIUS[k]) for k, R in enumerate(bench.R_PORES)
             for p in bench.PRESSURES]
    systems = [cd.DFTSystem(model, cd.Uniform1DSphr((p, bench.T_ISO), [model.stable_density(p, bench.T_ISO, [1.0])],
                                                     [0.0, R], N), cd.Steele(["graphite"])) for R, p, N in specs]
    for sy in systems:
        cd.dFdrho_res(sy, cd.initialize_profiles(sy))   # the plans' device profiles
    plans = (ctypes.c_void_p * len(systems))(*[sy._plan.value for sy in systems])
    out = {}
    for v in (0, 1, 2):
        cd.tuning("radial_dmma", v)
        ms = ctypes.c_double()
        _lib.check(lib.cdft_batch_time_stage(plans, len(systems), 0, 50, ctypes.byref(ms)))
        out[v] = ms.value
    for sy in systems:
        sy.close()
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=None)
    args = ap.parse_args()
    import cdft_b200 as cd
    defaults = {k: cd.tuning(k) for k in ("pers_warp_aa_max_elem", "fft3d_tma", "fft3d_fused_phi", "radial_dmma")}
    res = {"isotherm64_ms_per_batch": sweep_isotherm(), "solutes3d_ms_per_functional_derivative": sweep_3d(),
           "radial_isotherm64_ms_per_dense_stage": sweep_radial()}
    for k, v in defaults.items():
        cd.tuning(k, v)
    iso = res["isotherm64_ms_per_batch"]
    best = {"pers_warp_aa_max_elem": min(iso, key=lambda v: iso[v]["us_per_critical_evaluation"])}
    d3 = res["solutes3d_ms_per_functional_derivative"]
    totals = {}
    for key, ms in d3.items():
        shape = key.split(" ", 2)[2]
        totals[shape] = totals.get(shape, 0.0) + ms
    shape = min(totals, key=totals.get)
    best["fft3d_tma"] = int(shape.split()[0].split("=")[1])
    best["fft3d_fused_phi"] = int(shape.split()[1].split("=")[1])
    rad = res["radial_isotherm64_ms_per_dense_stage"]
    best["radial_dmma"] = min(rad, key=rad.get)
    res["best"] = best
    res["defaults_compiled"] = defaults
    res["when"] = time.strftime("%Y-%m-%dT%H:%M:%SZ", time.gmtime())
    line = json.dumps(res, default=str)
    print(line)
    if args.out:
        with open(args.out, "w") as f:
            f.write(line + "\n")


if __name__ == "__main__":
    main()
