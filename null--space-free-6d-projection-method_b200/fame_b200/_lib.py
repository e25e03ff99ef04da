"""ctypes binding of libfame_b200.so (the C ABI declared in include/fame.h).

The library is required: importing this module raises if it is missing, and
there is no CPU fallback anywhere in the package.
"""
from __future__ import annotations

import ctypes as C
import os

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libfame_b200.so")

FAME_OK = 0
FAME_ERR_INVALID = 1
FAME_ERR_CUDA = 2
FAME_ERR_OOM = 3
FAME_ERR_NOT_CONVERGED = 4
FAME_ERR_NONFINITE = 5
FAME_ERR_BUDGET = 6
FAME_ERR_SINGULAR = 7
FAME_ERR_UNSUPPORTED = 8
FAME_ERR_BREAKDOWN = 9

FAME_F64, FAME_F32 = 0, 1
FAME_MASS_SCALAR, FAME_MASS_FULL3, FAME_MASS_COL3, FAME_MASS_COLS12 = 0, 1, 2, 3
FAME_KRINV_EXPLICIT, FAME_KRINV_NESTED = 0, 1
FAME_PREC_FP64, FAME_PREC_MIXED = 0, 1


class fame_basis_info(C.Structure):
    _fields_ = [("NF", C.c_longlong), ("N", C.c_int), ("nsingular", C.c_int),
                ("minQq", C.c_double), ("minAbsDetV1", C.c_double), ("kLift", C.c_double * 6),
                ("pivot", C.c_int)]


class fame_krinv_opts(C.Structure):
    _fields_ = [("kind", C.c_int), ("prec_mode", C.c_int), ("tolCG", C.c_double),
                ("maxitCG", C.c_int), ("tolKr", C.c_double), ("tolM", C.c_double),
                ("maxitKr", C.c_int), ("maxitM", C.c_int), ("epsC", C.c_double),
                ("useKrPreconditioner", C.c_int), ("tolInner32", C.c_double),
                ("maxRefine", C.c_int), ("checkEvery", C.c_int), ("verifyTrueResidual", C.c_int),
                ("useGraphs", C.c_int), ("mhatPreconditioner", C.c_int), ("passColumns", C.c_int),
                ("refineTarget", C.c_double)]


class fame_krinv_stats(C.Structure):
    _fields_ = [("inverseCalls", C.c_longlong), ("totalIterations", C.c_longlong),
                ("maxIterations", C.c_longlong), ("maxRelativeResidual", C.c_double),
                ("massSolveCalls", C.c_longlong), ("totalMassIterations", C.c_longlong),
                ("refineSteps", C.c_longlong), ("fp32Iterations", C.c_longlong),
                ("massApplies", C.c_longlong), ("totalInverseSeconds", C.c_double)]


class fame_lanczos_info(C.Structure):
    _fields_ = [("steps", C.c_int), ("restarts", C.c_int), ("converged", C.c_int),
                ("nconv", C.c_int), ("maxWantedResidual", C.c_double)]


class fame_osi_stats(C.Structure):
    _fields_ = [("topApplications", C.c_longlong), ("minresIterations", C.c_longlong),
                ("cycles", C.c_longlong), ("maxTrueRelres", C.c_double), ("failures", C.c_int),
                ("plateauAccepts", C.c_int)]


P = C.c_void_p
I = C.c_int
LL = C.c_longlong
D = C.c_double

# name -> (argtypes)
SIGNATURES = {
    "fame_version": [],
    "fame_ctx_create": [I, C.POINTER(P)],
    "fame_ctx_destroy": [P],
    "fame_ctx_set_stream": [P, P],
    "fame_ctx_use_own_stream": [P],
    "fame_ctx_sync": [P],
    "fame_applyMij_fft": [P, I, P, P, P, I, I],
    "fame_mass_create": [P, I, P, C.POINTER(P)],
    "fame_mass_destroy": [P],
    "fame_mass_apply": [P, I, P, P, I, I],
    "fame_selftest_bounded_wait": [P, C.c_uint],
    "fame_applyMij_rank1_exact": [P, P, P, LL, P, P, I],
    "fame_rank1_exact_fft_scatter": [P, P, I, P, LL, LL, P],
    "fame_rank1_exact_ifft_gather": [P, P, I, P, LL, LL, P],
    "fame_apply_V_blockdiag": [P, P, P, P, P, P, P, P, LL, I, P],
    "fame_apply_VH_blockdiag": [P, P, P, P, P, P, P, P, LL, I, P],
    "fame_solveV1_blockdiag": [P, P, P, P, P, P, P, LL, I, P],
    "fame_solveV1H_blockdiag": [P, P, P, P, P, P, P, LL, I, P],
    "fame_basis_create": [P, I, C.POINTER(D), C.POINTER(D), C.POINTER(P)],
    "fame_basis_destroy": [P],
    "fame_basis_info_get": [P, C.POINTER(fame_basis_info)],
    "fame_basis_get": [P, I, P],
    "fame_krinv_default_opts": [C.POINTER(fame_krinv_opts)],
    "fame_krinv_create": [P, P, C.POINTER(fame_krinv_opts), C.POINTER(P)],
    "fame_krinv_destroy": [P],
    "fame_krinv_apply": [P, P, P, I],
    "fame_krinv_stats_get": [P, C.POINTER(fame_krinv_stats)],
    "fame_krinv_stats_reset": [P],
    "fame_device_trim_memory": [I],
    "fame_lanczos": [P, I, D, I, I, P, C.POINTER(D), P, C.POINTER(fame_lanczos_info)],
    "fame_rayleigh_ritz": [P, P, P, I, C.POINTER(D), C.POINTER(D)],
    "fame_osi_create": [P, P, D, D, D, I, C.POINTER(P)],
    "fame_osi_destroy": [P],
    "fame_osi_apply": [P, P, P, I],
    "fame_osi_eigs": [P, I, D, I, I, P, C.POINTER(D), P, C.POINTER(fame_lanczos_info)],
    "fame_osi_stats_get": [P, C.POINTER(fame_osi_stats)],
    "fame_apply_K_original": [P, P, P, I],
    "fame_start_vector": [P, C.c_ulonglong, LL, P],
    "fame_apply_Mhat_C_scalar_compact": [P, P, P, P, I],
    "fame_apply_Mhat_C_scalar_compact_noalloc": [P, P, P, P, I],
    "fame_recover_eigvecs": [P, P, P, I, D, I, I, P, P, C.POINTER(I), C.POINTER(D)],
    "fame_fourier_diagnostics": [P, P, P, C.POINTER(D), I, C.POINTER(D), C.POINTER(D), C.POINTER(D)],
    "fame_reconstruct_direct": [P, P, P, LL, P, LL, P],
    "fame_reconstruct_direct_grid": [P, P, P, I, P, I, P, I, P],
    "fame_reconstruct_direct_grid_3xtf32": [P, P, P, I, P, I, P, I, P],
    "fame_reconstruct_direct_grid_fields": [P, P, I, P, I, P, I, P, I, I, P],
    "fame_taylor_on_blocks": [P, P, P, LL, P, LL, I, P, P, I, C.POINTER(D), P],
    "fame_taylor_on_blocks_3xtf32": [P, P, P, LL, P, LL, I, P, P, I, C.POINTER(D), P],
    "fame_mass_adjoint": [P, P, I, P, I, C.POINTER(D)],
    "fame_yee_lwrq_metrics": [P, P, P, P, I, D, C.POINTER(D), I, D, D, D, C.POINTER(D), C.POINTER(D), C.POINTER(D)],
    "fame_solve_batch": [I, I, C.POINTER(I), C.POINTER(P), C.POINTER(D), C.POINTER(D),
                         C.POINTER(fame_krinv_opts), I, D, I, I, C.c_ulonglong, C.POINTER(D),
                         C.POINTER(fame_lanczos_info), C.POINTER(I)],
    "fame_solve_batch_each": [I, I, C.POINTER(I), C.POINTER(P), C.POINTER(D), C.POINTER(D),
                              C.POINTER(fame_krinv_opts), I, D, I, I, C.c_ulonglong, C.POINTER(D),
                              C.POINTER(fame_lanczos_info), C.POINTER(I)],
}


class FameError(RuntimeError):
    """A non-zero status from the C ABI (``status`` holds the FAME_ERR_* code)."""

    def __init__(self, status: int, message: str):
        super().__init__(message)
        self.status = status


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError("libfame_b200.so is not built (%s); run build.py in the package directory"
                          % LIB_PATH)
    lib = C.CDLL(LIB_PATH)
    for name, argt in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.argtypes = argt
        fn.restype = C.c_int
    lib.fame_status_string.argtypes = [C.c_int]
    lib.fame_status_string.restype = C.c_char_p
    lib.fame_last_error.argtypes = []
    lib.fame_last_error.restype = C.c_char_p
    lib.fame_kernel_launches.argtypes = []
    lib.fame_kernel_launches.restype = C.c_longlong
    return lib


lib = _load()


def check(status: int):
    if status != FAME_OK:
        raise FameError(status, lib.fame_last_error().decode())
    return status


def call(name: str, *args):
    return check(getattr(lib, name)(*args))
