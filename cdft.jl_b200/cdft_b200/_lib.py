"""ctypes binding of libcdft_b200.so (include/cdft_b200.h).

The library is built in-tree (``python -m cdft_b200.build`` or
``__graft_entry__.build()``) and loaded from this directory only; there is no
fallback implementation: every compute call goes through the CUDA library.
"""
import ctypes
import os

import numpy as np

MAX_NC = 4
MAX_ASSOC = 8
MAX_SITES = 8
MAX_M = 16

OK = 0
E_INVALID = -1
E_CUDA = -2
E_UNSUPPORTED = -3
E_BUDGET = -4

COORD_CART, COORD_SPH, COORD_CYL = 0, 1, 2
PREC_FP64, PREC_MIXED = 0, 1
NOALLOC_MAX_N = 4096
NOALLOC_MAX_ELEM = 8192
ENGINE_AUTO, ENGINE_GRID, ENGINE_PERSISTENT = 0, 1, 2

LIB_NAME = "libcdft_b200.so"
# CDFT_B200_LIB selects another build of the library (the Julia shim honours the same variable)
LIB_PATH = os.environ.get("CDFT_B200_LIB") or os.path.join(os.path.dirname(os.path.abspath(__file__)), LIB_NAME)

# every symbol declared in include/cdft_b200.h
EXPORTED = [
    "cdft_plan_create", "cdft_plan_destroy",
    "cdft_functional_derivative", "cdft_functional_derivative_dev", "cdft_ddft_rhs", "cdft_ddft_rhs_dev", "cdft_bulk_density", "cdft_saturation_pure", "cdft_phi_field",
    "cdft_free_energy_res", "cdft_phi_pointwise", "cdft_free_energy_res_grad", "cdft_grad_params", "cdft_grad_params_ext",
    "cdft_converge", "cdft_converge_dev",
    "cdft_batch_converge", "cdft_batch_converge_dev",
    "cdft_plan_set_stream", "cdft_batch_time_stage", "cdft_functional_derivative_noalloc",
    "cdft_tuning_get", "cdft_tuning_set", "cdft_batch_integrals",
    "cdft_launch_count", "cdft_last_error", "cdft_version",
]


class AssocPair(ctypes.Structure):
    _fields_ = [
        ("icomp", ctypes.c_int), ("jcomp", ctypes.c_int),
        ("isite", ctypes.c_int), ("jsite", ctypes.c_int),
        ("n_ia", ctypes.c_int), ("n_jb", ctypes.c_int),
        ("eps_ab", ctypes.c_double), ("kappa_ab", ctypes.c_double),
    ]


class SystemDesc(ctypes.Structure):
    _fields_ = [
        ("nd", ctypes.c_int),
        ("ngrid", ctypes.c_int * 3),
        ("bounds", (ctypes.c_double * 2) * 3),
        ("coord", ctypes.c_int),
        ("nc", ctypes.c_int),
        ("m", ctypes.c_double * MAX_NC),
        ("hsd", ctypes.c_double * MAX_NC),
        ("sigma", ctypes.c_double * (MAX_NC * MAX_NC)),
        ("eps", ctypes.c_double * (MAX_NC * MAX_NC)),
        ("L", ctypes.c_double),
        ("T", ctypes.c_double),
        ("n_assoc", ctypes.c_int),
        ("assoc", AssocPair * MAX_ASSOC),
        ("mu_res_plus_ln_rhob", ctypes.c_double * MAX_NC),
        ("vext", ctypes.POINTER(ctypes.c_double)),
        ("precision", ctypes.c_int),
    ]


class SolverOpts(ctypes.Structure):
    _fields_ = [
        ("m", ctypes.c_int),
        ("maxit", ctypes.c_int),
        ("rtol", ctypes.c_double), ("atol", ctypes.c_double), ("beta", ctypes.c_double),
        ("picard_maxit", ctypes.c_int),
        ("picard_beta", ctypes.c_double), ("picard_rtol", ctypes.c_double), ("picard_atol", ctypes.c_double),
        ("time_budget_s", ctypes.c_double),
        ("iters_per_launch", ctypes.c_int),
        ("engine", ctypes.c_int),
        ("mixed_switch_rtol", ctypes.c_double),
        ("snapshot_every", ctypes.c_int),
        ("snapshot", ctypes.c_void_p),
        ("snapshot_user", ctypes.c_void_p),
    ]


# void (*)(void* user, int system, int evaluations, const double* rho)
SNAPSHOT_FN = ctypes.CFUNCTYPE(None, ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_double))


class Result(ctypes.Structure):
    _fields_ = [
        ("idid", ctypes.c_int), ("errcode", ctypes.c_int),
        ("iterations", ctypes.c_int), ("evaluations", ctypes.c_int),
        ("resnorm", ctypes.c_double), ("tol", ctypes.c_double),
        ("history", ctypes.POINTER(ctypes.c_double)),
        ("history_cap", ctypes.c_int), ("history_len", ctypes.c_int),
    ]


class CDFTError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"cdft_b200 error {code}: {msg}")
        self.code = code


_lib = None


def load(path=LIB_PATH):
    """Load the CUDA library; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise ImportError(f"{path} is missing: build the CUDA library first (cdft_b200.build.build())")
    lib = ctypes.CDLL(path)
    P = ctypes.c_void_p
    dp = ctypes.POINTER(ctypes.c_double)
    lib.cdft_plan_create.argtypes = [ctypes.POINTER(SystemDesc), ctypes.POINTER(P)]
    lib.cdft_plan_destroy.argtypes = [P]
    lib.cdft_functional_derivative.argtypes = [P, dp, dp]
    lib.cdft_functional_derivative_dev.argtypes = [P, P, P]
    lib.cdft_ddft_rhs.argtypes = [P, P, P]
    lib.cdft_ddft_rhs_dev.argtypes = [P, P, P]
    lib.cdft_phi_field.argtypes = [P, P, P]
    lib.cdft_bulk_density.argtypes = [ctypes.POINTER(SystemDesc), ctypes.c_int, P, P, ctypes.c_int, P, P]
    lib.cdft_saturation_pure.argtypes = [ctypes.POINTER(SystemDesc), ctypes.c_int, P, P, P, P, P]
    lib.cdft_free_energy_res.argtypes = [P, dp, dp]
    lib.cdft_phi_pointwise.argtypes = [P, dp, ctypes.c_int, dp, dp]
    lib.cdft_free_energy_res_grad.argtypes = [P, dp, dp]
    lib.cdft_grad_params.argtypes = [P, dp, dp, dp, dp]
    lib.cdft_grad_params_ext.argtypes = [P, dp, dp, dp, dp, dp]
    lib.cdft_converge.argtypes = [P, dp, ctypes.POINTER(SolverOpts), ctypes.POINTER(Result)]
    lib.cdft_converge_dev.argtypes = [P, P, ctypes.POINTER(SolverOpts), ctypes.POINTER(Result)]
    lib.cdft_batch_converge.argtypes = [ctypes.POINTER(P), ctypes.c_int, ctypes.POINTER(dp),
                                        ctypes.POINTER(SolverOpts), ctypes.POINTER(Result)]
    lib.cdft_batch_converge_dev.argtypes = [ctypes.POINTER(P), ctypes.c_int, ctypes.POINTER(P),
                                            ctypes.POINTER(SolverOpts), ctypes.POINTER(Result)]
    lib.cdft_plan_set_stream.argtypes = [P, P]
    lib.cdft_batch_time_stage.argtypes = [ctypes.POINTER(P), ctypes.c_int, ctypes.c_int, ctypes.c_int, dp]
    lib.cdft_functional_derivative_noalloc.argtypes = [ctypes.POINTER(SystemDesc), P, P, P]
    lib.cdft_batch_integrals.argtypes = [ctypes.POINTER(P), ctypes.c_int, ctypes.POINTER(P), ctypes.c_int, dp]
    lib.cdft_tuning_get.argtypes = [ctypes.c_char_p, ctypes.POINTER(ctypes.c_int)]
    lib.cdft_tuning_set.argtypes = [ctypes.c_char_p, ctypes.c_int]
    lib.cdft_launch_count.argtypes = [ctypes.c_int]
    lib.cdft_launch_count.restype = ctypes.c_longlong
    lib.cdft_last_error.argtypes = [ctypes.c_char_p, ctypes.c_size_t]
    lib.cdft_version.restype = ctypes.c_char_p
    for name in EXPORTED:
        getattr(lib, name).restype = getattr(lib, name).restype or ctypes.c_int
    _lib = lib
    return lib


def check(rc):
    if rc != OK:
        buf = ctypes.create_string_buffer(512)
        _lib.cdft_last_error(buf, 512)
        raise CDFTError(rc, buf.value.decode(errors="replace"))
    return rc


def dptr(a):
    """Pointer to a C-contiguous float64 numpy array."""
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
