"""ctypes binding of the C++ CPU restatement of converge! (``cpu_converge.cpp``).

Test infrastructure and the timed CPU baseline: the compiled counterpart of the NumPy
oracle for 1D Cartesian systems, run with OpenMP over state points.  Systems are
described from the oracle's ``functional.DFTSystem`` in the library's own C layout
(``include/cdft_b200.h``: ``cdft_system_desc``, ``cdft_solver_opts``, ``cdft_result``).

    python oracle/cpu.py          # build oracle/libcdft_cpu.so
"""
import ctypes
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "cpu_converge.cpp")
OUT = os.path.join(HERE, "libcdft_cpu.so")
HEADER = os.path.join(HERE, "..", "include", "cdft_b200.h")
# x86-64-v3 (AVX2, FMA): every host of a B200 node has it; the library is built once
# and runs on the host cores of the GPU machines as well
FLAGS = ["-O3", "-std=c++17", "-march=x86-64-v3", "-fopenmp", "-fPIC", "-shared"]

MAX_NC, MAX_ASSOC = 4, 8


class AssocPair(ctypes.Structure):
    _fields_ = [("icomp", ctypes.c_int), ("jcomp", ctypes.c_int), ("isite", ctypes.c_int), ("jsite", ctypes.c_int),
                ("n_ia", ctypes.c_int), ("n_jb", ctypes.c_int), ("eps_ab", ctypes.c_double), ("kappa_ab", ctypes.c_double)]


class SystemDesc(ctypes.Structure):
    _fields_ = [
        ("nd", ctypes.c_int), ("ngrid", ctypes.c_int * 3), ("bounds", (ctypes.c_double * 2) * 3),
        ("coord", ctypes.c_int), ("nc", ctypes.c_int), ("m", ctypes.c_double * MAX_NC),
        ("hsd", ctypes.c_double * MAX_NC), ("sigma", ctypes.c_double * (MAX_NC * MAX_NC)),
        ("eps", ctypes.c_double * (MAX_NC * MAX_NC)), ("L", ctypes.c_double), ("T", ctypes.c_double),
        ("n_assoc", ctypes.c_int), ("assoc", AssocPair * MAX_ASSOC),
        ("mu_res_plus_ln_rhob", ctypes.c_double * MAX_NC), ("vext", ctypes.POINTER(ctypes.c_double)),
        ("precision", ctypes.c_int),
    ]


class SolverOpts(ctypes.Structure):
    _fields_ = [
        ("m", ctypes.c_int), ("maxit", ctypes.c_int), ("rtol", ctypes.c_double), ("atol", ctypes.c_double),
        ("beta", ctypes.c_double), ("picard_maxit", ctypes.c_int), ("picard_beta", ctypes.c_double),
        ("picard_rtol", ctypes.c_double), ("picard_atol", ctypes.c_double), ("time_budget_s", ctypes.c_double),
        ("iters_per_launch", ctypes.c_int), ("engine", ctypes.c_int), ("mixed_switch_rtol", ctypes.c_double),
        ("snapshot_every", ctypes.c_int), ("snapshot", ctypes.c_void_p), ("snapshot_user", ctypes.c_void_p),
    ]


class Result(ctypes.Structure):
    _fields_ = [
        ("idid", ctypes.c_int), ("errcode", ctypes.c_int), ("iterations", ctypes.c_int),
        ("evaluations", ctypes.c_int), ("resnorm", ctypes.c_double), ("tol", ctypes.c_double),
        ("history", ctypes.POINTER(ctypes.c_double)), ("history_cap", ctypes.c_int), ("history_len", ctypes.c_int),
    ]


def build(force=False, verbose=False):
    deps = [SRC, HEADER]
    if not force and os.path.exists(OUT) and all(os.path.getmtime(d) <= os.path.getmtime(OUT) for d in deps):
        return OUT
    cmd = ["g++"] + FLAGS + ["-o", OUT, SRC]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    return OUT


_LIB = None


def load():
    global _LIB
    if _LIB is None:
        if not os.path.exists(OUT):
            raise RuntimeError(f"{OUT} is not built: run python oracle/cpu.py")
        lib = ctypes.CDLL(OUT)
        lib.cdft_cpu_functional_derivative.argtypes = [ctypes.POINTER(SystemDesc), ctypes.c_void_p, ctypes.c_void_p]
        lib.cdft_cpu_batch_converge.argtypes = [ctypes.POINTER(SystemDesc), ctypes.c_int, ctypes.c_void_p,
                                                ctypes.POINTER(SolverOpts), ctypes.POINTER(Result), ctypes.c_int]
        lib.cdft_cpu_max_threads.restype = ctypes.c_int
        lib.cdft_cpu_set_wb_closed.argtypes = [ctypes.c_int]
        lib.cdft_cpu_set_wb_closed.restype = None
        _LIB = lib
    return _LIB


def fn_pairs(so):
    from .functional import assoc_site_pairs
    return assoc_site_pairs(so.model)


def desc_of(so):
    """cdft_system_desc of an oracle functional.DFTSystem (1D Cartesian); keeps the
    V_ext array alive on the returned object."""
    st = so.structure
    d = SystemDesc()
    d.nd = 1
    d.ngrid[0] = st.ngrid[0]
    d.bounds[0][0], d.bounds[0][1] = st.bounds[0]
    d.coord = 0
    nc = so.nc
    d.nc = nc
    for i in range(nc):
        d.m[i] = so.m[i]
        d.hsd[i] = so.hsd[i]
        d.mu_res_plus_ln_rhob[i] = so.chem_pot_res_dens[i]
        for j in range(nc):
            d.sigma[i * nc + j] = so.model.sigma_ij[i, j]
            d.eps[i * nc + j] = so.eps_ij[i, j]
    d.L = so.L
    d.T = st.T
    if len(fn_pairs(so)) > 1:
        raise NotImplementedError("the C++ restatement covers the one-pair association path")
    d.n_assoc = len(so.model.assoc)
    if so.model.assoc:
        ic, jc, eab, kab = so.model.assoc[0]
        d.assoc[0] = AssocPair(ic, jc, 0, 1, 1, 1, eab, kab)
    vext = None if so.vext is None else np.ascontiguousarray(so.vext, dtype=np.float64)
    d.vext = vext.ctypes.data_as(ctypes.POINTER(ctypes.c_double)) if vext is not None else None
    d._keep = vext
    return d


def solver_opts(beta=1e-2, tol=1e-4, anderson_start=1e-1, anderson_m=5, maxit=10000):
    """converge!'s keywords mapped onto AASol as __AASol does (converge.jl:3-13)."""
    o = SolverOpts()
    o.m, o.maxit, o.rtol, o.atol, o.beta = anderson_m, maxit, tol, tol, beta
    o.picard_maxit, o.picard_beta, o.picard_rtol, o.picard_atol = maxit, beta, anderson_start, anderson_start
    return o


def functional_derivative(so, rho):
    d = desc_of(so)
    rho = np.ascontiguousarray(rho, dtype=np.float64)
    out = np.empty_like(rho)
    rc = load().cdft_cpu_functional_derivative(ctypes.byref(d), rho.ctypes.data, out.ctypes.data)
    if rc:
        raise RuntimeError(f"cdft_cpu_functional_derivative: {rc}")
    return out


def batch_converge(systems, rhos, nthreads=0, history_cap=0, **solver):
    """Converge the oracle systems' profiles in place on `nthreads` host threads (0: all);
    returns the cdft_result records."""
    n = len(systems)
    descs = (SystemDesc * n)()
    keep = []
    for k, so in enumerate(systems):
        d = desc_of(so)
        keep.append(d._keep)
        descs[k] = d
    for r in rhos:
        assert r.flags.c_contiguous and r.dtype == np.float64
    ptrs = (ctypes.c_void_p * n)(*[r.ctypes.data for r in rhos])
    res = (Result * n)()
    hist = []
    if history_cap:
        for k in range(n):
            h = np.zeros(history_cap)
            hist.append(h)
            res[k].history = h.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
            res[k].history_cap = history_cap
    o = solver_opts(**solver)
    rc = load().cdft_cpu_batch_converge(descs, n, ptrs, ctypes.byref(o), res, nthreads)
    if rc:
        raise RuntimeError(f"cdft_cpu_batch_converge: {rc}")
    return [res[k] for k in range(n)], hist


def set_wb_closed(closed):
    """Evaluate the reference's closed White-Bear bracket everywhere (True) or the series
    form near n3 = 0 (False, the default)."""
    load().cdft_cpu_set_wb_closed(1 if closed else 0)


def max_threads():
    return load().cdft_cpu_max_threads()


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
