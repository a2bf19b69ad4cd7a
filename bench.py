"""Benchmark of the converge! hot path on B200.

Workload (default): the batched adsorption isotherm -- PC-SAFT methane at
150 K in graphite slit pores, 8 pore widths 2-8 nm x 8 pressures log-spaced
1e3-1e7 Pa = 64 state points with uneven grids (100..400 points, linear in the
width), Anderson m=5, beta=0.1, tol=1e-10, all converged together through
cdft_batch_converge.  A step converges all 64 systems from their initial
profiles.  Metric: state points per second (whole job, all ranks).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--precision fp64|mixed]
    python bench.py --impl reference ...   # the reference's algorithm compiled for the host cores

Multi-GPU (torchrun): the job is one 64-point isotherm per rank (pressures shifted by
0.1 % per isotherm; weak scaling), its state points split across ranks by longest
processing time first on their estimated cost (cdft_b200.shard); every rank converges
its share as one batch with no collective on the data path, the timed region is
bracketed by a barrier, the device time is the max over ranks, and rank 0 gathers
(adsorption, Omega_ex, status, rho) of every state point afterwards.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "cdft.jl_b200"))
sys.path.insert(0, ROOT)

T_ISO = 150.0
WIDTHS = np.linspace(2e-9, 8e-9, 8)
PRESSURES = np.logspace(3, 7, 8)
N_OF_WIDTH = [int(round(100 + 300 * k / 7)) for k in range(8)]
SOLVER = dict(beta=0.1, tol=1e-10, anderson_m=5, maxit=10000)
METHANE = dict(m=[1.0], sigma=[3.7039], epsilon=[150.03])
# DRAM bytes (read + write) per launch of the dominant kernel, from one ncu capture of the
# same command (dram__bytes_read.sum + dram__bytes_write.sum; the summaries and commands are
# in profiles/): the isotherm's persistent_kernel, one launch per step.
ISO_TRAFFIC_BYTES = 1.915904e6 + 0.0
FP64_PEAK_NOMINAL_TFLOPS = 37.0   # HGX B200 FP64 / FP64 tensor (datasheet); no measured FP64 peak exists for this pool


def isotherm_specs(rank=0):
    """(width, pressure, N) of the 64 state points; ranks > 0 shift pressures by 0.1% per rank."""
    out = []
    for k, H in enumerate(WIDTHS):
        for p in PRESSURES:
            out.append((float(H), float(p) * (1 + 1e-3 * rank), N_OF_WIDTH[k]))
    return out


def job_specs(world):
    """All state points of a job on `world` ranks: one isotherm per rank."""
    return [s for r in range(world) for s in isotherm_specs(r)]


def max_over_ranks(value, dist, device):
    """Max of a per-rank time over all ranks (all_reduce MAX), then a barrier."""
    import torch
    t = torch.tensor([float(value)], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    dist.barrier()
    return float(t.item())


def whole_job_rate(units_per_rank, world, ms_max):
    """Units per second of the whole job: every rank's units over the slowest rank's time."""
    return units_per_rank * world / (ms_max * 1e-3)


def _views_of(flat, arrays):
    """Views of one flat device tensor shaped like each of ``arrays``, back to back."""
    out, o = [], 0
    for a in arrays:
        out.append(flat[o:o + a.size].view(a.shape))
        o += a.size
    return out


def _device_views(arrays):
    """All ``arrays`` in one device allocation: (the flat tensor, a view per array)."""
    import torch
    flat = torch.from_numpy(np.concatenate([np.ascontiguousarray(a).ravel() for a in arrays])).cuda()
    return flat, _views_of(flat, arrays)


def build_systems(specs, precision, bulk="host"):
    """The isotherm's DFT systems.  bulk = "host": the stable bulk root of every state point
    from the host solver (equal to the committed oracle fixture's to 1 ulp: the headline's
    inputs); "device": from cdft_bulk_density in one launch (the user's whole pipeline).
    The two differ in the last bits, and a few state points' evaluation counts are chaotic
    in those bits (the same aasol on the CPU: 93-853 evaluations for the 8 nm / 10 MPa pore
    over +-6e-13 relative changes of rho_b)."""
    import cdft_b200 as cd
    model = cd.PCSAFT(["methane"], **METHANE)
    s = model.sigma[0]
    systems, rho0 = [], []
    if bulk == "device":
        rbs = cd.bulk_density(model, [p for _, p, _ in specs], T_ISO, [1.0], "stable")
    else:
        rbs = [model.stable_density(p, T_ISO, [1.0]) for _, p, _ in specs]
    for (H, p, N), rb in zip(specs, rbs):
        st = cd.Uniform1DCart((p, T_ISO), [rb], [0.7 * s, H - 0.7 * s], N)
        sy = cd.DFTSystem(model, st, cd.Steele(["graphite"], H), cd.DFTOptions(precision))
        systems.append(sy)
        rho0.append(cd.initialize_profiles(sy))
    return systems, rho0


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except FileNotFoundError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            return json.load(f)
    return None


def accuracy_vs_oracle(systems, rhos):
    """Largest relative errors of converged isotherm results against the oracle fixture
    of the same 64 state points (tests/golden/c3_isotherm64.npz: the CPU oracle converged
    to 1e-13): profiles, adsorption and the excess grand potential Omega_ex (the
    numerator of surface_tension)."""
    import cdft_b200 as cd
    path = os.path.join(ROOT, "tests", "golden", "c3_isotherm64.npz")
    if not os.path.exists(path):
        return None
    f = np.load(path)
    off = f["offsets"]
    e_rho = e_ads = e_om = 0.0
    for k, (sy, r) in enumerate(zip(systems, rhos)):
        ref = f["rho"][off[k]:off[k + 1]]
        e_rho = max(e_rho, float(np.max(np.abs(r[0] / ref - 1))))
        e_ads = max(e_ads, abs(cd.adsorption(sy, r)[0] / f["adsorption"][k] - 1))
        e_om = max(e_om, abs(cd.surface_tension(sy, r) / f["omega_ex"][k] - 1))
    return {"rho_rel_err_max": e_rho, "adsorption_rel_err_max": e_ads, "omega_ex_rel_err_max": e_om,
            "oracle": "tests/golden/c3_isotherm64.npz (CPU oracle, FP64, tol 1e-13)"}


def run_ours(args, rank, world, local_rank):
    import ctypes
    import torch
    import cdft_b200 as cd
    from cdft_b200 import _lib

    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    from cdft_b200 import shard
    lib = _lib.load()
    all_specs = job_specs(world)
    parts = shard.lpt_partition([shard.estimated_cost(N) for _, _, N in all_specs], world)
    mine = parts[rank]
    specs = [all_specs[i] for i in mine]
    stream = torch.cuda.Stream()
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")   # > 126 MB L2
    method = cd.AASol.for_system(None, **SOLVER)

    def timed(fn, steps, warmup):
        for _ in range(warmup):
            fn()
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        total = 0.0
        for _ in range(steps):
            flush.fill_(1.0)                       # evict the previous step's data from L2 (untimed)
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            fn()
            e1.record(stream)
            e1.synchronize()
            total += e0.elapsed_time(e1)
        torch.cuda.synchronize()
        if dist:
            total = max_over_ranks(total, dist, "cuda")
        return total / steps

    def device_isotherm(precision, steps, warmup):
        """Converge the 64 systems from device-resident initial profiles
        (cdft_batch_converge_dev); CUDA events on the plans' stream."""
        systems, rho0 = build_systems(specs, precision)
        n = len(systems)
        for sy in systems:
            _lib.check(lib.cdft_plan_set_stream(sy._plan, ctypes.c_void_p(stream.cuda_stream)))
        opts = method.c_opts(engine=args.engine)
        plans = (ctypes.c_void_p * n)(*[sy._plan.value for sy in systems])
        # the 64 profiles are views of one device allocation: a step restores all of them
        # with one copy
        init_flat, _ = _device_views(rho0)
        work_flat = torch.empty_like(init_flat)
        work_dev = _views_of(work_flat, rho0)
        ptrs = (ctypes.c_void_p * n)(*[t.data_ptr() for t in work_dev])
        results = (_lib.Result * n)()

        def step():
            with torch.cuda.stream(stream):
                work_flat.copy_(init_flat, non_blocking=True)
            _lib.check(lib.cdft_batch_converge_dev(plans, n, ptrs, ctypes.byref(opts), results))

        cd.launch_count(reset=True)
        ms = timed(step, steps, warmup)
        launches = cd.launch_count(reset=True)
        evals = [results[i].evaluations for i in range(n)]
        errc = [results[i].errcode for i in range(n)]
        rho_out = [t.cpu().numpy() for t in work_dev]
        return dict(systems=systems, rho0=rho0, plans=plans, ms=ms, evals=evals, errc=errc, rho=rho_out,
                    launches=int(round(launches * steps / (steps + warmup))))

    with ClockSampler(local_rank) as clk:
        run = device_isotherm(args.precision, args.steps, args.warmup)
    systems, rho0, plans, n = run["systems"], run["rho0"], run["plans"], len(run["systems"])
    iters, errc, ms_dev = run["evals"], run["errc"], run["ms"]

    # e2e through the public host API: host profiles in, converged host profiles out
    host_in = [r.copy() for r in rho0]
    host_work = [np.empty_like(r) for r in rho0]

    def step_e2e():
        for w, i in zip(host_work, host_in):
            w[...] = i
        cd.batch_converge(systems, host_work, method=method, engine=args.engine)

    ms_e2e = timed(step_e2e, max(1, args.steps), 1)

    # the user's whole isotherm: adsorption(model, surface, p, T) builds a DFTSystem per state
    # point (src/methods/adsorption.jl:48-65): plan creation (device tables), initial profiles,
    # the batched converge and the host copies; host wall clock around synchronised work
    setup_evals = []

    def step_setup():
        sy, r0 = build_systems(specs, args.precision, bulk="device")
        rs = cd.batch_converge(sy, r0, method=method, engine=args.engine)
        setup_evals[:] = [x.evaluations for x in rs]
        for x in sy:
            x.close()

    step_setup()
    torch.cuda.synchronize()
    t_set = []
    for _ in range(max(1, min(args.steps, 3))):
        t0 = time.perf_counter()
        step_setup()
        torch.cuda.synchronize()
        t_set.append(time.perf_counter() - t0)
    ms_setup = 1e3 * float(np.mean(t_set))

    # host gather of every state point's results to rank 0 (outside the timed region)
    records = [(float(cd.adsorption(sy, r)[0]), float(cd.surface_tension(sy, r)), int(e), r)
               for sy, r, e in zip(systems, run["rho"], errc)]
    gathered = shard.gather_results(dist, rank, world, mine, records, len(all_specs))
    accuracy = accuracy_vs_oracle(systems, run["rho"]) if world == 1 else None
    mixed = None
    if rank == 0 and args.precision == "fp64" and args.mixed:
        mr = device_isotherm("mixed", max(2, args.steps // 4), 2)
        mixed = {"value": round(n / (mr["ms"] * 1e-3), 3), "unit": "state points/s",
                 "ms_per_step": round(mr["ms"], 4), "speedup_vs_fp64": round(ms_dev / mr["ms"], 3),
                 "evaluations_per_system": {"min": min(mr["evals"]), "max": max(mr["evals"]),
                                            "mean": float(np.mean(mr["evals"]))},
                 "errcodes": sorted(set(mr["errc"])),
                 "accuracy_vs_oracle": accuracy_vs_oracle(mr["systems"], mr["rho"])}
        for sy in mr["systems"]:
            sy.close()

    # convolution stage alone (one launch covering all systems), timed with CUDA events
    ms_conv = ctypes.c_double()
    _lib.check(lib.cdft_batch_time_stage(plans, n, 0, 200, ctypes.byref(ms_conv)))
    ms_phi = ctypes.c_double()
    _lib.check(lib.cdft_batch_time_stage(plans, n, 1, 200, ctypes.byref(ms_phi)))
    flops_conv = sum(2.0 * s.nc * 6 * s.ngrid[0] ** 2 for s in systems)
    conv_tflops = flops_conv / (ms_conv.value * 1e-3) / 1e12
    # the dominant kernel of a step: the persistent converge kernel (one launch per step) or,
    # in the grid engine, the convolutions; algorithmic work = 2 convolution stages per evaluation
    step_flops = sum(2.0 * 2.0 * s.nc * 6 * s.ngrid[0] ** 2 * ev for s, ev in zip(systems, iters))
    achieved = step_flops / (ms_dev * 1e-3) / 1e12
    plain = plain_fp64_gpu(specs) if (rank == 0 and args.plain) else None
    total_units = len(all_specs)
    value = total_units / (ms_dev * 1e-3)
    h2d = sum(r.nbytes for r in rho0)
    line = None
    if rank == 0:
        line = {
            "metric": "state points/s (64-point slit-pore adsorption isotherm, batched converge!)",
            "value": round(value, 3),
            "unit": "state points/s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": round(ms_dev, 4),
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f64" if args.precision == "fp64" else "f32 conv+Phi / f64 solver",
            "data": "synthetic: seeded isotherm state points, PC-SAFT methane parameters",
            "config": {
                "workload": "isotherm64: methane 150 K, graphite slit pores 2-8 nm x 1e3-1e7 Pa, N=100..400",
                "state_points": total_units, "systems_per_gpu": n, "grid_points": sum(s.ngrid[0] for s in systems),
                "sharding": {"ranks": world, "partition": "LPT on N^2 per state point",
                             "balance_max_over_mean": round(shard.balance(
                                 parts, [shard.estimated_cost(N) for _, _, N in all_specs]), 4),
                             "gathered_state_points": len(gathered),
                             "gathered_errcodes": sorted(set(g[2] for g in gathered))},
                "solver": SOLVER, "precision": args.precision, "engine": args.engine,
                "l2": "flushed between steps (256 MB write, untimed)",
                "evaluations_per_system": {"min": min(iters), "max": max(iters), "mean": float(np.mean(iters))},
                "errcodes": sorted(set(errc)),
            },
            "e2e": {"value": round(total_units / (ms_e2e * 1e-3), 3), "unit": "state points/s",
                    "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": h2d},
            "e2e_with_setup": {
                "value": round(n / (ms_setup * 1e-3), 3), "unit": "state points/s", "ms_per_step": round(ms_setup, 2),
                "how": ("bulk densities of the 64 state points in one device launch, 64 x (DFTSystem: bulk "
                        "mu_res on the host, plan creation with its device kernel tables; initialize_profiles) "
                        "+ batched converge with host arrays, host wall clock"),
                "evaluations_per_system": {"min": int(min(setup_evals)), "max": int(max(setup_evals)),
                                           "mean": float(np.mean(setup_evals))}},
            "gpu_launches": run["launches"],
            "roofline": {
                "kernel": ("persistent_kernel (whole batched converge, 1 launch per step; circulant "
                           "convolutions on the FP64 tensor cores, mma.sync m8n8k4 f64)" if args.engine != "grid"
                           else "grid engine (14 launches per evaluation)"),
                "bound": "tensor",
                "achieved": round(achieved, 3),
                "peak": FP64_PEAK_NOMINAL_TFLOPS,
                "peak_source": "nominal HGX B200 FP64 tensor (of nominal: MEASURED_PEAKS.json has no FP64 figure)",
                "unit": "TFLOP/s",
                "frac": round(achieved / FP64_PEAK_NOMINAL_TFLOPS, 4),
                "traffic": ISO_TRAFFIC_BYTES if args.engine != "grid" else None,
                "traffic_unit": "bytes per launch (ncu, profiles/isotherm64_fp64_persistent_kernel.md)",
                "algorithmic_flops_per_launch": step_flops,
                "stage_conv1d": {"ms_per_launch": round(ms_conv.value, 5), "tflops": round(conv_tflops, 3),
                                 "algorithmic_flops_per_launch": flops_conv},
                "stage_phi_ms_per_launch": round(ms_phi.value, 5),
            },
            "clocks": clk.summary(),
        }
        if accuracy is not None:
            line["accuracy_vs_oracle"] = accuracy
        if mixed is not None:
            line["mixed_isotherm"] = mixed
    if rank == 0 and plain is not None:
        line["plain_fp64_gpu_path"] = plain
    if rank == 0 and args.radial:
        line["radial_isotherm"] = radial_isotherm()
    if rank == 0 and args.with3d:
        line["solutes3d"] = {str(N): solutes3d(N, plain=args.plain) for N in args.grid3d}
    if args.cpu_baseline and rank == 0:
        line["cpu_baseline"] = cpu_baseline(specs, budget_s=args.cpu_budget)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return line


# spherical pore radii 1-3 nm (diameters 2-6 nm) and their point counts.  A 4 nm radius is left
# out: its 7.2e5 Pa state point sits at the capillary transition, where aasol from the bulk
# profile does not converge within maxit for any beta in 0.02-0.1 or m in 5-10.
R_PORES = np.linspace(1e-9, 3e-9, 8)
N_OF_RADIUS = [int(round(100 + 200 * k / 7)) for k in range(8)]


def radial_isotherm(steps=3, warmup=2):
    """Second 1D workload: the isotherm in spherical graphite pores (Uniform1DSphr with the
    curved Steele wall, steele.jl:111-143), 8 radii x the 8 pressures = 64 state points,
    N = 100..300 linear in the radius, on the grid engine.  Plans of one radius share one
    device operator buffer, so each radius's weighted densities are one FP64 tensor-core
    GEMM over its state points (radial_dmma = 1) instead of 8 matrix-vector products
    (radial_dmma = 0).  Reports the batched converge with both, the dense stage alone
    (operator bytes per launch / time, against the measured copy bandwidth), the plan
    creation time of the 64 state points and the two modes' largest profile difference."""
    import ctypes
    import torch
    import cdft_b200 as cd
    from cdft_b200 import _lib
    lib = _lib.load()
    model = cd.PCSAFT(["methane"], **METHANE)
    specs = [(float(R), float(p), N_OF_RADIUS[k]) for k, R in enumerate(R_PORES) for p in PRESSURES]
    rbs = [model.stable_density(p, T_ISO, [1.0]) for _, p, _ in specs]
    t0 = time.perf_counter()
    systems = [cd.DFTSystem(model, cd.Uniform1DSphr((p, T_ISO), [rb], [0.0, R], N), cd.Steele(["graphite"]))
               for (R, p, N), rb in zip(specs, rbs)]
    ms_plans = 1e3 * (time.perf_counter() - t0)
    rho0 = [cd.initialize_profiles(sy) for sy in systems]
    n = len(systems)
    stream = torch.cuda.Stream()
    for sy in systems:
        _lib.check(lib.cdft_plan_set_stream(sy._plan, ctypes.c_void_p(stream.cuda_stream)))
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    opts = cd.AASol.for_system(None, **SOLVER).c_opts(engine="grid")
    plans = (ctypes.c_void_p * n)(*[sy._plan.value for sy in systems])
    init_flat, _ = _device_views(rho0)
    work_flat = torch.empty_like(init_flat)
    work_dev = _views_of(work_flat, rho0)
    ptrs = (ctypes.c_void_p * n)(*[t.data_ptr() for t in work_dev])
    results = (_lib.Result * n)()

    def step():
        with torch.cuda.stream(stream):
            work_flat.copy_(init_flat, non_blocking=True)
        _lib.check(lib.cdft_batch_converge_dev(plans, n, ptrs, ctypes.byref(opts), results))

    # operator bytes one dense-stage launch reads: each radius's N x N operators (6 fields)
    # once per column tile of 8 state points, plus the inputs and outputs
    op_bytes = 0
    for k in range(len(R_PORES)):
        N = N_OF_RADIUS[k]
        tiles = (len(PRESSURES) + 7) // 8
        op_bytes += tiles * 6 * N * N * 8 + len(PRESSURES) * 2 * 6 * N * 8
    flops = sum(2.0 * 6 * N * N for _, _, N in specs)
    peak = (measured_peaks() or {}).get("hbm_gbs")
    out = {"workload": "radial isotherm64: methane 150 K, spherical graphite pores r = 1-3 nm x 1e3-1e7 Pa, "
                       "N=100..300, grid engine", "solver": SOLVER,
           "plan_creation_ms_64": round(ms_plans, 1),
           "plan_creation_how": "64 DFTSystem constructions; the dense operators are built once per radius "
                                "(O(N^3) on the host) and shared by the plans of that radius"}
    profiles = {}
    default = cd.tuning("radial_dmma")   # the tensor-core GEMM (1: 8-row CTAs, 2: 16-row CTAs, same bits)
    try:
        for mode in (default, 0):
            cd.tuning("radial_dmma", mode)
            for _ in range(warmup):
                step()
            torch.cuda.synchronize()
            total = 0.0
            for _ in range(steps):
                flush.fill_(1.0)
                torch.cuda.synchronize()
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                step()
                e1.record(stream)
                e1.synchronize()
                total += e0.elapsed_time(e1)
            ms = total / steps
            evals = [results[i].evaluations for i in range(n)]
            errc = sorted(set(results[i].errcode for i in range(n)))
            profiles[mode] = [t.cpu().numpy() for t in work_dev]
            ms_stage = ctypes.c_double()
            _lib.check(lib.cdft_batch_time_stage(plans, n, 0, 200, ctypes.byref(ms_stage)))
            key = "dmma_gemm" if mode else "warp_rows"
            out[key] = {"value": round(n / (ms * 1e-3), 3), "unit": "state points/s", "ms_per_step": round(ms, 4),
                        "evaluations_per_system": {"min": min(evals), "max": max(evals),
                                                   "mean": float(np.mean(evals))},
                        "errcodes": errc,
                        "dense_stage_ms_per_launch": round(ms_stage.value, 5)}
            if mode:
                gbs = op_bytes / (ms_stage.value * 1e-3) / 1e9
                out[key]["roofline"] = {
                    "kernel": f"dense_group_kernel (mma.sync m8n8k4 f64, 8 state points per column tile, "
                              f"{8 * mode} rows per CTA)",
                    "bound": "hbm", "achieved": round(gbs, 1), "peak": peak, "unit": "GB/s",
                    "frac": round(gbs / peak, 4) if peak else None,
                    "algorithmic_bytes_per_launch": op_bytes,
                    "tflops": round(flops / (ms_stage.value * 1e-3) / 1e12, 3),
                    "note": "the operators (18 MB per stage) stay in the 126 MB L2 between back-to-back "
                            "launches, so the fraction can exceed 1 of the HBM copy bandwidth"}
    finally:
        cd.tuning("radial_dmma", default)
    out["speedup_dmma_over_warp_rows"] = round(out["warp_rows"]["ms_per_step"] / out["dmma_gemm"]["ms_per_step"], 3)
    out["max_rel_diff_between_modes"] = float(max(np.max(np.abs(a / b - 1)) for a, b in zip(profiles[default], profiles[0])))
    for sy in systems:
        sy.close()
    return out


ARGON = dict(m=[1.0], sigma=[3.4], epsilon=[120.0])
T_3D = 100.0
SOLVER_3D = dict(beta=0.1, tol=1e-10, anderson_m=10, maxit=2000)


def _solutes3d_system(N, precision):
    import cdft_b200 as cd
    model = cd.PCSAFT(["argon"], **ARGON)
    s = model.sigma[0]
    box = 16 * s
    rb = 0.021e30 / cd.N_A
    st = cd.Uniform3DCart((1e5, T_3D), [rb], [0.0, box], N)
    centres = cd.HardSphereSolutes.seeded(27, 1.5 * s, box, 2 * box / N, seed=0)
    return cd.DFTSystem(model, st, cd.HardSphereSolutes(centres, 1.5 * s), cd.DFTOptions(precision))


# Algorithmic HBM bytes per grid point per Anderson iteration of the 3D path
# (nc = 1, NF = 9, m = 10, one V_ext), each array read or written once per stage:
#   (a) weighted densities  s (nc + (NF-1) nc)          FP64  72
#   (b) Phi / dPhi          s (2 NF nc)                        144
#   (c) adjoint + EL        s (NF nc + nc) + 8 (V_ext)          88
#   (d) Anderson vectors    8 nc (2 m + 6)                     208
# = 512 B in FP64 (s = 8), 364 B mixed (s = 4); FFT-internal passes are excluded.
BYTES_3D_ITER = {"fp64": 512, "mixed": 364}
# DRAM bytes per point of one FP64 Anderson iteration as measured (ncu, dram__bytes_read.sum +
# dram__bytes_write.sum over one iteration's 20 launches at 128^3: 2.494e9 B / 128^3)
TRAFFIC_3D_ITER_BYTES_PER_POINT = 1189.3
# What the FFT pipeline of one functional derivative moves per point (x, y, z passes
# of rho, the 8 convolved fields and the 8 dPhi/dn fields, Phi and the EL output;
# the half spectrum holds 16 B per (N/2+1)/N point, counted as 8 B per real point):
#   forward rho: x 8+8, y 16, z + multiply 8+64                    = 104
#   inverse of the 8 convolved fields: y 128, x 64+64              = 256
#   Phi: read 9 fields 72, write 8 gradients 64                    = 136
#   forward of the 8 gradients: x 64+64, y 128                     = 256
#   z adjoint 64+8, inverse y 16, x 8+8                            = 104
#   Euler-Lagrange output: rho, V_ext, adjoint in, G(rho) out      =  32
# = 888 B/point in FP64; mixed: FFT and Phi arrays in FP32, the rest FP64.
BYTES_3D_PIPE = {"fp64": 888, "mixed": (104 + 256 + 136 + 256 + 104) // 2 + 32}


def solutes3d_run(N, precision, reps=2):
    """One precision of the 3D configuration at N^3: converged from the initial
    profile through cdft_converge_dev (device-resident rho), CUDA-event timed."""
    import ctypes
    import torch
    import cdft_b200 as cd
    from cdft_b200 import _lib
    sy = _solutes3d_system(N, precision)
    rho0 = cd.initialize_profiles(sy)
    stream = torch.cuda.Stream()
    lib = _lib.load()
    _lib.check(lib.cdft_plan_set_stream(sy._plan, ctypes.c_void_p(stream.cuda_stream)))
    method = cd.AASol.for_system(None, **SOLVER_3D)
    opts = method.c_opts(engine="grid")
    init = torch.from_numpy(rho0).cuda()
    work = torch.empty_like(init)
    res = _lib.Result()

    def run():
        with torch.cuda.stream(stream):
            work.copy_(init)
        _lib.check(lib.cdft_converge_dev(sy._plan, ctypes.c_void_p(work.data_ptr()), ctypes.byref(opts),
                                         ctypes.byref(res)))

    run()   # warm-up (graph capture)
    torch.cuda.synchronize()
    cd.launch_count(reset=True)
    times = []
    for _ in range(reps):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        run()
        e1.record(stream)
        e1.synchronize()
        times.append(e0.elapsed_time(e1))
    launches = cd.launch_count(reset=True) // reps
    ms = float(np.mean(times))
    evals = res.evaluations
    ips = evals / (ms * 1e-3)
    ms_eval = ctypes.c_double()
    plans = (ctypes.c_void_p * 1)(sy._plan.value)
    _lib.check(lib.cdft_batch_time_stage(plans, 1, 3, 20, ctypes.byref(ms_eval)))
    rho = work.cpu().numpy()
    omega = cd.surface_tension(sy, rho)   # F k_B T - sum mu int rho + p V: excess grand potential, J
    fluid = sy.vext == 0
    sy.close()
    peaks = measured_peaks()
    peak = peaks["hbm_gbs"] if peaks else 6650.0
    achieved = BYTES_3D_ITER[precision] * N ** 3 * ips / 1e9
    pipe = BYTES_3D_PIPE[precision] * N ** 3 / (ms_eval.value * 1e-3) / 1e9
    src = "MEASURED_PEAKS.json hbm_gbs (of measured)" if peaks else "fallback 6650 GB/s (of fallback)"
    out = {
        "iterations_per_s": round(ips, 2), "ms_per_converge": round(ms, 3), "evaluations": evals,
        "errcode": res.errcode, "ms_per_iteration": round(ms / evals, 4), "gpu_launches_per_converge": launches,
        "functional_derivative_ms": round(ms_eval.value, 4),
        "roofline": {
            "bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "peak_source": src,
            "unit": "GB/s", "frac": round(achieved / peak, 4),
            "traffic": (TRAFFIC_3D_ITER_BYTES_PER_POINT * N ** 3 if precision == "fp64" else None),
            "traffic_unit": ("DRAM bytes per iteration, all of its launches (ncu at 128^3 in the Anderson phase, "
                             "per point scaled to N^3; profiles/solutes3d_128_fp64_kernels.md)"),
            "algorithmic_bytes_per_point_iteration": BYTES_3D_ITER[precision]},
        "functional_derivative_pipeline": {
            "bytes_per_point": BYTES_3D_PIPE[precision], "achieved_gbs": round(pipe, 1),
            "frac": round(pipe / peak, 4)},
    }
    return out, rho, omega, fluid


def solutes3d(N=128, reps=2, plain=True):
    """3D configuration: PC-SAFT argon, 100 K, rho_b = 0.021 A^-3, periodic cubic box of
    edge 16 sigma on N^3 points, 27 hard spherical solutes of radius 1.5 sigma at
    non-overlapping positions (numpy default_rng(0), centre gaps >= 3 sigma + 2 cells),
    Anderson m = 10, beta = 0.1, tol = 1e-10.  FP64 and mixed, each converged from the
    initial profile; the mixed profile and excess grand potential are compared with
    the FP64 ones (relative errors; rho over the fluid, V_ext = 0)."""
    r64, rho64, om64, fluid = solutes3d_run(N, "fp64", reps)
    r32, rho32, om32, _ = solutes3d_run(N, "mixed", reps)
    out = {
        "workload": f"solutes3d: argon 100 K, {N}^3 periodic box edge 16 sigma, 27 hard solutes r=1.5 sigma",
        "solver": SOLVER_3D, "fp64": r64, "mixed": r32,
        "mixed_vs_fp64": {
            "rho_rel_err_max_fluid": float(np.max(np.abs(rho32[fluid] / rho64[fluid] - 1))),
            "omega_rel_err": abs(om32 / om64 - 1),
            "speedup_converge": round(r64["ms_per_converge"] / r32["ms_per_converge"], 3),
            "speedup_per_iteration": round(r64["ms_per_iteration"] / r32["ms_per_iteration"], 3),
        },
    }
    if plain:
        p = plain_fp64_gpu_3d(N)
        out["plain_fp64_gpu_path"] = p
        out["speedup_vs_plain_fp64_gpu"] = {
            "fp64_per_iteration": round(p["ms_per_iteration"] / r64["ms_per_iteration"], 3),
            "mixed_per_iteration": round(p["ms_per_iteration"] / r32["ms_per_iteration"], 3),
            "fp64_converge": round(1e3 * p["seconds"] / r64["ms_per_converge"], 3),
            "mixed_converge": round(1e3 * p["seconds"] / r32["ms_per_converge"], 3),
        }
    return out


def run_3d_only(args):
    """--only3d: the 3D configuration alone at one size and precision (profiling runs)."""
    import torch
    torch.cuda.set_device(0)
    N = args.grid3d[0]
    for _ in range(max(0, args.warmup - 1)):
        solutes3d_run(N, args.precision, reps=1)
    r, _, _, _ = solutes3d_run(N, args.precision, reps=max(1, args.steps))
    return {"metric": "3D iterations/s (solutes3d)", "value": r["iterations_per_s"], "unit": "iterations/s",
            "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": r["ms_per_converge"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if args.precision == "fp64" else "f32 FFT+Phi / f64 solver",
            "data": "synthetic: seeded solute positions",
            "config": {"workload": f"solutes3d {N}^3", "solver": SOLVER_3D}, "solutes3d": r}


# ---------------------------------------------------------------------------
# The plain FP64 GPU path of the 3D configuration, built with the reference's structure on
# cuFFT (torch.fft) and PyTorch: every convolution copies its input into a complex buffer,
# runs a forward and an inverse C2C FFT and keeps the real part (convolve!,
# src/utils/integrals.jl:88-96) -- rho is transformed again for every field; Phi's gradient
# comes from automatic differentiation of the pointwise f_res (models.jl:131-186; reverse
# mode, one pass, where the reference's default runs one forward pass per field); aasol
# keeps its vectors on the device and solves the small least-squares problem and the QR
# downdate on the host (anderson.jl:386-416,552-583), one device-host round trip per step.
# The comparison arm for "plain FP64 GPU path" of the 3D configuration.
# ---------------------------------------------------------------------------
def plain3d_params(sy):
    """The scalars and arrays of a one-component 3D system that the plain path needs."""
    st = sy.structure
    lb, ub = st.bounds[0]
    return dict(N=st.ngrid[0], box=ub - lb, L=sy.L, d=float(sy.size[0] / sy.L), m=float(sy.model.m[0]),
                s=float(sy.model.sigma_ij[0, 0] / sy.L), eps=float(sy.model.eps_ij[0, 0]), T=st.conditions[1],
                vext=np.ascontiguousarray(sy.vext[0]), cprd=float(sy.chempot_res[0] + np.log(st.rho_bulk[0])))


def plain3d_functional(prm, device="cuda"):
    """G(x) = clamp(mu_res + ln rho_b - dF/drho[exp x] - V_ext) of the plain path (GFix!,
    converge.jl:108-153), on torch tensors of shape (N, N, N), grid order (z, y, x)."""
    import torch
    from cdft_b200.thermo import _A, _B
    N, L, d, m = prm["N"], prm["L"], prm["d"], prm["m"]
    s3 = prm["s"] ** 3
    eT = prm["eps"] / prm["T"]
    NA = 6.02214076e23 * L ** 3
    dev = device
    w1 = torch.tensor(np.fft.fftfreq(N) * N / prm["box"] * L, dtype=torch.float64, device=dev)
    KZ, KY, KX = torch.meshgrid(w1, w1, w1, indexing="ij")
    wb = torch.sqrt(KX * KX + KY * KY + KZ * KZ)
    zero = wb == 0
    safe = torch.where(zero, torch.ones_like(wb), wb)
    two_pi = 2 * np.pi

    def k_dz(R):
        return (torch.where(zero, torch.full_like(wb, 2 * R), 2 * torch.sin(safe * R) / safe) / two_pi).to(torch.complex128)

    def k_z2dz(R):
        return (torch.where(zero, torch.full_like(wb, 4 * np.pi * R ** 3 / 3),
                            4 * np.pi / safe ** 3 * (torch.sin(safe * R) - R * safe * torch.cos(safe * R)))
                / two_pi ** 3).to(torch.complex128)

    def k_vec(R):
        core = 4 * np.pi / safe ** 3 * (torch.sin(safe * R) - R * safe * torch.cos(safe * R))
        return [torch.complex(torch.zeros_like(wb), torch.where(zero, torch.full_like(wb, 4 * np.pi * R), od * core))
                / two_pi ** 3 for od in (KX, KY, KZ)]

    R = lambda w: two_pi * w * d
    psi = 1.3862
    K = [k_dz(R(0.5)), k_z2dz(R(0.5))] + k_vec(R(0.5)) + [k_z2dz(R(1.0)), k_dz(R(1.0)), k_z2dz(R(psi))]
    sign = [1, 1, -1, -1, -1, 1, 1, 1]   # vector fields enter the adjoint with -= (fields.jl:50-61)
    A = torch.tensor(np.asarray(_A), dtype=torch.float64, device=dev)
    B = torch.tensor(np.asarray(_B), dtype=torch.float64, device=dev)
    wbs = torch.tensor([(j + 1.0) * (j + 3.0) / (j + 2.0) for j in range(16)], dtype=torch.float64, device=dev)
    vext = torch.from_numpy(prm["vext"]).to(dev)
    cprd = prm["cprd"]

    def conv(f, k):   # convolve!: C2C forward and inverse FFT, real part
        return torch.fft.ifftn(torch.fft.fftn(f.to(torch.complex128)) * k).real

    def f_res(n):
        n0 = n[1] * m / d
        n1 = 0.5 * n[1] * m
        n2 = np.pi * n[1] * m * d
        nv1 = [n[2 + k] * m / d for k in (1, 2, 3)]
        nv2 = [-2 * np.pi * n[2 + k] * m for k in (1, 2, 3)]
        n3 = n[2] * m
        nv1v2 = nv1[0] * nv2[0] + nv1[1] * nv2[1] + nv1[2] * nv2[2]
        nv2sq = nv2[0] * nv2[0] + nv2[1] * nv2[1] + nv2[2] * nv2[2]
        dn = 1 - n3
        log1dn = torch.log(torch.abs(dn))
        small = torch.abs(n3) < 0.05
        n3s = torch.where(small, torch.full_like(n3, 0.5), n3)   # closed form only where it is used
        closed = log1dn / (12 * np.pi * n3s * n3s) + 1 / (12 * np.pi * n3s * dn * dn)
        ser = torch.zeros_like(n3) + wbs[15]
        for j in range(14, -1, -1):
            ser = ser * n3 + wbs[j]
        bkt = torch.where(small, ser / (12 * np.pi), closed)
        res = -n0 * log1dn + (n1 * n2 - nv1v2) / dn + (n2 * n2 * n2 / 3 - n2 * nv2sq) * bkt
        z3 = m * n[6] / 8   # chain (PCSAFT.jl:123-144); (m - 1) = 0 for argon
        z2 = m * n[6] / d / 8
        inv1 = 1 / (1 - z3)
        ydd = inv1 + 1.5 * d * z2 * inv1 * inv1 + 0.5 * d * d * z2 * z2 * inv1 ** 3
        res = res - n[0] * (m - 1) * torch.log(torch.abs(ydd * (n[7] / (2 * d)) / n[0]))
        rz = n[8] * (3 / (4 * psi ** 3 * np.pi)) / d ** 3
        eta = m * rz * d ** 3 * np.pi / 6
        cij = rz * rz * m * m * s3
        s1, s2 = cij * eT, cij * eT * eT
        e2 = eta * eta
        C1 = 1 + m * (8 * eta - 2 * e2) / (1 - eta) ** 4 + (1 - m) * (20 * eta - 27 * e2 + 12 * eta * e2 - 2 * e2 * e2) / (
            (1 - eta) ** 2 * (2 - eta) ** 2)
        c1 = (m - 1) / m
        c2 = c1 * (m - 2) / m
        I1 = torch.zeros_like(eta)
        I2 = torch.zeros_like(eta)
        for k in range(6, -1, -1):
            I1 = I1 * eta + (A[k, 0] + c1 * A[k, 1] + c2 * A[k, 2])
            I2 = I2 * eta + (B[k, 0] + c1 * B[k, 1] + c2 * B[k, 2])
        return res - 2 * np.pi * I1 * s1 - np.pi * m * I2 * s2 / C1

    def gfix(lnx):   # GFix!: rho = exp(x); ln G = mu + ln rho_b - dF/drho - V_ext, clamp (converge.jl:108-153)
        rho = torch.exp(lnx)
        n = [(rho * NA).requires_grad_(True)] + [(conv(rho, k) * NA).requires_grad_(True) for k in K]
        phi = f_res(n).sum()
        g = torch.autograd.grad(phi, n)
        out = g[0].detach()
        for gf, k, sg in zip(g[1:], K, sign):
            out = out + sg * conv(gf.detach(), k)
        return torch.clamp(cprd - out - vext, -100.0, 100.0)

    return gfix


def plain_aasol(gfix, x0, m=10, beta=0.1, tol=1e-10, anderson_start=0.1, maxit=2000):
    """aasol (anderson.jl:301-443; picard_maxit = maxit, picard_beta = beta, Picard
    tolerances anderson_start) with the vectors on the device -- the history Q and DG as
    m rows of n contiguous values, the columns of the reference's column-major matrices --
    and the small triangular solve and the downdate's Householder QR (LAPACK through
    numpy, downdate_aaqr!, anderson.jl:552-583) on the host.  Returns (x, evaluations, ok)."""
    import torch
    import scipy.linalg
    shape = x0.shape
    n = x0.numel()

    def G(x):
        return ((1 - beta) * x + beta * gfix(x.view(shape)).reshape(-1))

    sol = x0.reshape(-1).clone()
    gx = G(sol)
    res = gx - sol
    resnorm = float(torch.linalg.norm(res))
    up, tolv, ptol = 1e4 * resnorm, tol * resnorm + tol, anderson_start * resnorm + anderson_start
    evals, k = 1, 0
    toosoon = resnorm <= tolv
    if not toosoon:   # Picard warm-up
        sol = gx.clone()
        for _ in range(maxit - 1):
            gx = G(sol)
            evals += 1
            res = gx - sol
            resnorm = float(torch.linalg.norm(res))
            if resnorm <= ptol or resnorm >= up:
                break
            sol = gx.clone()
        toosoon = resnorm <= tolv
    Qt = torch.zeros((m, n), dtype=torch.float64, device=x0.device)
    DGt = torch.zeros((m, n), dtype=torch.float64, device=x0.device)
    Rm = np.zeros((m, m))

    def point(gx, sol, res):
        g = G(sol)
        r = g - sol
        return g, g - gx, r - res, r, float(torch.linalg.norm(r))

    dg = df = None
    if not toosoon:
        sol = gx.clone()
        k = 1
        gx, dg, df, res, resnorm = point(gx, sol, res)
        evals += 1
    while k < 2 * maxit and resnorm > tolv and not toosoon and resnorm < up:
        kk = k + 1
        if kk > m + 1:   # BuildDG!
            DGt = torch.roll(DGt, -1, dims=0)
            DGt[m - 1] = dg
        else:
            DGt[kk - 2] = dg
        kq0 = k - 1
        if kq0 == 0:
            nv = float(torch.linalg.norm(df))
            Rm[0, 0] = nv
            Qt[0] = df / nv
        else:
            if kq0 > m - 1:
                Qx, Rd = np.linalg.qr(Rm[:, 1:m])
                Rm[:] = 0.0
                Rm[:m - 1, :m - 1] = Rd
                Qt[:m - 1] = torch.from_numpy(np.ascontiguousarray(Qx.T)).to(Qt.device) @ Qt
                Qt[m - 1] = 0.0
            kq = min(kq0, m - 1)
            Qk = Qt[:kq]
            h1 = Qk @ df   # CGS2 (Orthogonalize!, anderson.jl:525-540)
            v = df - h1 @ Qk
            h2 = Qk @ v
            v = v - h2 @ Qk
            nv = float(torch.linalg.norm(v))
            Rm[:kq, kq] = (h1 + h2).cpu().numpy()
            Rm[kq, kq] = nv
            Qt[kq] = v / nv
        mk = min(m, k)
        tres = (Qt[:mk] @ res).cpu().numpy()
        theta = scipy.linalg.solve_triangular(Rm[:mk, :mk], tres, lower=False)
        sol = gx - torch.from_numpy(theta).to(gx.device) @ DGt[:mk]
        k += 1
        gx, dg, df, res, resnorm = point(gx, sol, res)
        evals += 1
    return sol.view(shape), evals, bool(resnorm <= tolv)


def plain_fp64_gpu_3d(N):
    """The reference-structured FP64 GPU path converging the 3D configuration: Anderson
    iterations per second (fixed-point evaluations over the CUDA-synchronised wall time of
    the whole solve) and its converged excess grand potential beside ours."""
    import torch
    import cdft_b200 as cd
    sy = _solutes3d_system(N, "fp64")
    prm = plain3d_params(sy)
    gfix = plain3d_functional(prm, "cuda")
    x0 = torch.log(torch.from_numpy(cd.initialize_profiles(sy)[0]).cuda())
    gfix(x0)   # warm-up (cuFFT plans, allocator)
    torch.cuda.synchronize()
    t = time.perf_counter()
    x, evals, ok = plain_aasol(gfix, x0, m=SOLVER_3D["anderson_m"], beta=SOLVER_3D["beta"],
                               tol=SOLVER_3D["tol"], maxit=SOLVER_3D["maxit"])
    torch.cuda.synchronize()
    dt = time.perf_counter() - t
    rho = torch.exp(x).cpu().numpy()[None]
    om_plain = float(cd.surface_tension(sy, rho))
    rho_ours = cd.initialize_profiles(sy)
    cd.converge(sy, rho_ours, method=cd.AASol.for_system(None, **SOLVER_3D))
    om_ours = float(cd.surface_tension(sy, rho_ours))
    sy.close()
    return {"iterations_per_s": round(evals / dt, 3), "ms_per_iteration": round(1e3 * dt / evals, 3),
            "evaluations": evals, "converged": ok, "seconds": round(dt, 3),
            "omega_ex_rel_diff_vs_ours": abs(om_plain / om_ours - 1),
            "rho_max_rel_diff_vs_ours": float(np.max(np.abs(rho / rho_ours - 1))),
            "how": ("reference structure on cuFFT + PyTorch: a C2C FFT pair per convolution (rho transformed "
                    "again for every field), autograd dPhi/dn, aasol with device vectors and a host-side "
                    "triangular solve / downdate QR; whole solve timed")}


def plain_fp64_gpu(specs):
    """The plain FP64 GPU path: the same 64 systems converged one converge! call at a
    time with per-stage kernels (the reference's CUDA path structure), wall time."""
    import torch
    import cdft_b200 as cd
    s64, r64 = build_systems(specs, "fp64")
    method = cd.AASol.for_system(None, **SOLVER)
    for s, r in zip(s64, r64):   # warm-up: every plan's CUDA graph is captured outside the timing
        cd.converge(s, r.copy(), method=method, engine="grid", keep_history=False)
    torch.cuda.synchronize()
    t = time.perf_counter()
    for s, r in zip(s64, r64):
        cd.converge(s, r.copy(), method=method, engine="grid", keep_history=False)
    dt = time.perf_counter() - t
    return {"ms": round(dt * 1e3, 2), "value": round(len(s64) / dt, 3), "unit": "state points/s",
            "how": "64 sequential cdft_converge calls, FP64, grid engine, host wall clock, graphs captured "
                   "in an untimed warm-up pass"}


def _oracle_isotherm_systems(specs):
    """The isotherm's state points as oracle systems (bulk density of the stable phase)."""
    sys.path.insert(0, ROOT)
    from oracle import functional as fn, pcsaft_bulk as pb
    om = pb.PCSAFTModel(["methane"], METHANE["m"], METHANE["sigma"], METHANE["epsilon"])
    s = om.sigma[0]
    out = []
    for H, p, N in specs:
        roots = []
        for ph in ("liquid", "vapour"):
            try:
                roots.append(pb.density(om, p, T_ISO, [1.0], ph))
            except RuntimeError:
                pass
        rb = roots[0]
        if len(roots) == 2 and abs(roots[0] / roots[1] - 1) > 1e-10:
            g = [pb.mu_total(om, [r], T_ISO)[0] for r in roots]
            rb = roots[0] if g[0] <= g[1] else roots[1]
        st = fn.Structure((p, T_ISO), [rb], [(0.7 * s, H - 0.7 * s)], (N,))
        out.append(fn.DFTSystem(om, st, [fn.SteeleWall.graphite(H)]))
    return out


def _cpu_isotherm_step(systems, rho0, threads):
    """One converge of all state points by the C++ restatement of the reference's
    converge! (oracle/cpu_converge.cpp) on `threads` host threads; seconds."""
    from oracle import cpu
    rhos = [r.copy() for r in rho0]
    t0 = time.perf_counter()
    res, _ = cpu.batch_converge(systems, rhos, nthreads=threads, **SOLVER)
    dt = time.perf_counter() - t0
    return dt, [r.errcode for r in res]


def cpu_baseline(specs, budget_s=20.0):
    """The reference's algorithm compiled for the host (C++ restatement, FFT convolutions,
    forward-mode dPhi/dn, aasol) on all host cores: whole 64-point isotherm per step,
    repeated while the budget lasts (at least once)."""
    from oracle import cpu
    cpu.build()
    cores = os.cpu_count() or 1
    systems = _oracle_isotherm_systems(specs)
    rho0 = [so.initialize_profiles() for so in systems]
    times = []
    while not times or (sum(times) < budget_s and len(times) < 5):
        dt, errc = _cpu_isotherm_step(systems, rho0, cores)
        times.append(dt)
    return {"value": round(len(specs) / float(np.mean(times)), 3), "unit": "state points/s", "cores": cores,
            "kind": "port", "errcodes": sorted(set(errc)),
            "sample": (f"all {len(specs)} isotherm state points per step, {len(times)} steps; C++17 OpenMP "
                       "restatement of converge! (oracle/cpu_converge.cpp: Bluestein-FFT convolutions, "
                       "forward-mode dual-number dPhi/dn, aasol), one thread per state point, FP64")}


def run_reference(args, rank, world):
    """--impl reference: the reference's converge! on the host cores.  Julia is not
    available, so this is the compiled restatement of the reference's algorithm
    (oracle/cpu_converge.cpp) on all host threads, each step the whole 64-point
    isotherm (the configuration of the GPU arm)."""
    if rank != 0:
        return None
    from oracle import cpu
    cpu.build()
    cores = os.cpu_count() or 1
    specs = isotherm_specs(0)
    systems = _oracle_isotherm_systems(specs)
    rho0 = [so.initialize_profiles() for so in systems]
    times = []
    for it in range(args.warmup + args.steps):
        dt, errc = _cpu_isotherm_step(systems, rho0, cores)
        if it >= args.warmup:
            times.append(dt)
    ms = 1e3 * float(np.mean(times))
    value = len(specs) / (ms * 1e-3)
    return {
        "impl": "reference",
        "metric": "state points/s (64-point slit-pore adsorption isotherm, batched converge!)",
        "value": round(value, 4),
        "unit": "state points/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(ms, 2),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic: seeded isotherm state points, PC-SAFT methane parameters",
        "config": {"workload": "isotherm64: methane 150 K, graphite slit pores 2-8 nm x 1e3-1e7 Pa, N=100..400",
                   "solver": SOLVER, "state_points_per_step": len(specs), "errcodes": sorted(set(errc))},
        "cpu_baseline": {"value": round(value, 4), "unit": "state points/s", "cores": cores, "kind": "port",
                         "sample": (f"all {len(specs)} state points per step on {cores} OpenMP threads; C++17 "
                                    "restatement of the reference's converge! (oracle/cpu_converge.cpp)")},
        "e2e": {"value": round(value, 4), "unit": "state points/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("--engine", default="auto", choices=["auto", "grid", "persistent"])
    ap.add_argument("--no-cpu-baseline", dest="cpu_baseline", action="store_false")
    ap.add_argument("--cpu-budget", type=float, default=15.0)
    ap.add_argument("--no-plain", dest="plain", action="store_false", help="skip the sequential FP64 comparison")
    ap.add_argument("--no-mixed", dest="mixed", action="store_false", help="skip the mixed-precision isotherm")
    ap.add_argument("--no-3d", dest="with3d", action="store_false", help="skip the 3D solutes configuration")
    ap.add_argument("--no-radial", dest="radial", action="store_false", help="skip the spherical-pore isotherm")
    ap.add_argument("--only-radial", action="store_true", help="run only the spherical-pore isotherm")
    ap.add_argument("--grid3d", type=int, nargs="+", default=[128, 256])
    ap.add_argument("--only3d", action="store_true",
                    help="run only the 3D solutes configuration (first --grid3d size, --precision)")
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local_rank = int(os.environ.get("LOCAL_RANK", 0))
    if args.impl == "reference":
        line = run_reference(args, rank, world)
    elif args.only3d:
        line = run_3d_only(args) if rank == 0 else None
    elif args.only_radial:
        line = {"radial_isotherm": radial_isotherm(max(1, args.steps), max(1, args.warmup))} if rank == 0 else None
    else:
        line = run_ours(args, rank, world, local_rank)
    if rank == 0 and line is not None:
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
