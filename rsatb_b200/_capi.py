"""ctypes binding of the C ABI in include/rsatb_b200.h.

The shared library is built in-tree (``python -m rsatb_b200.build``) at
``rsatb_b200/_lib/librsatb_b200.so``.  There is no fallback: if the library
is missing or a call fails, an exception says so.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "_lib" / "librsatb_b200.so"

# rsatb_status
SUCCESS = 0
STATUS_NAMES = {
    0: "Success", 1: "InvalidArgument", 2: "FastPathRejected", 3: "RankBreakdown",
    4: "NotPositiveDefinite", 5: "NearSingular", 6: "NumericalFailure", 16: "CudaError",
    17: "OutOfMemory", 18: "NotSupported", 19: "Diverged", 20: "Interrupted",
}
# rsatb_dtype
F64, F32, C128, C64 = 0, 1, 2, 3
# rsatb_form
FORM_ORTHOGONAL, FORM_SANDWICH, FORM_SOLVE = 0, 1, 2
# rsatb_kpm_kernel
KPM_NONE, KPM_JACKSON, KPM_COSTAPER, KPM_VPTAPER = 0, 1, 2, 3
# rsatb_random_kind
RANDOM_PHASE, RANDOM_RADEMACHER, RANDOM_UNIFORM = 0, 1, 2
# rsatb_bsr_create flags
BSR_DEVICE_POINTERS, BSR_IMAGINARY_UNIT = 1, 2


class RsatbError(RuntimeError):
    """A C-ABI call returned a non-zero status."""

    def __init__(self, status: int, message: str):
        self.status = status
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")


class ChebOp(C.Structure):
    _fields_ = [("form", C.c_int), ("H", C.c_void_p), ("Z", C.c_void_p), ("ZH", C.c_void_p),
                ("center", C.c_double), ("half_width", C.c_double), ("S", C.c_void_p),
                ("cg_tol", C.c_double), ("cg_max_iter", C.c_int)]


class IsqrtOptions(C.Structure):
    _fields_ = [("precision", C.c_int), ("max_iter", C.c_int), ("max_fp64_iter", C.c_int),
                ("tol", C.c_double), ("accept", C.c_double), ("workspace_bytes", C.c_size_t),
                ("no_graph", C.c_int), ("tc_kernel", C.c_int), ("n_tiles", C.c_int),
                ("tile_n_pad", C.c_void_p), ("tile_nt", C.c_void_p)]


class IsqrtStats(C.Structure):
    _fields_ = [("chunks", C.c_int), ("low_iterations", C.c_int), ("fp64_iterations", C.c_int),
                ("n_failed", C.c_int), ("max_residual", C.c_double), ("low_flops", C.c_double),
                ("fp64_flops", C.c_double), ("useful_flops", C.c_double),
                ("gemm_launches", C.c_int64), ("low_ms", C.c_double), ("fp64_ms", C.c_double)]


class FftchebStats(C.Structure):
    _fields_ = [("sections", C.c_int), ("fft_chunks", C.c_int64), ("recurrence_ms", C.c_double),
                ("transform_ms", C.c_double), ("store_bytes", C.c_size_t)]


class AdjointStats(C.Structure):
    _fields_ = [("checkpoint_stride", C.c_int), ("segments", C.c_int),
                ("forward_ms", C.c_double), ("backward_ms", C.c_double),
                ("panels_held", C.c_int)]


class NsRefineOptions(C.Structure):
    _fields_ = [("tol", C.c_double), ("sptol", C.c_double), ("maxit", C.c_int),
                ("route", C.c_int)]


class NsRefineReport(C.Structure):
    _fields_ = [("steps", C.c_int), ("converged", C.c_int), ("hit_maxiter", C.c_int),
                ("diverged", C.c_int), ("last_advance_propagated", C.c_int),
                ("residual", C.c_double), ("applied_residual", C.c_double),
                ("nnz_blocks", C.c_int64), ("reforms", C.c_int), ("propagations", C.c_int)]


class LanczosOptions(C.Structure):
    _fields_ = [("steps", C.c_int), ("tol", C.c_double), ("max_matvecs", C.c_int),
                ("seed", C.c_uint64)]


class LanczosResult(C.Structure):
    _fields_ = [("theta_min", C.c_double), ("theta_max", C.c_double),
                ("res_min", C.c_double), ("res_max", C.c_double),
                ("matvecs", C.c_int), ("converged", C.c_int)]


# rsatb_ns_precision
NS_FP64, NS_TF32X3, NS_TF32 = 0, 1, 2

_lib = None

# name -> (restype, argtypes)
_vp, _i, _d, _u, _i64, _u64, _sz = (C.c_void_p, C.c_int, C.c_double, C.c_uint, C.c_int64,
                                    C.c_uint64, C.c_size_t)
_PD = C.POINTER(C.c_double)
SIGNATURES = {
    "rsatb_last_error": (C.c_char_p, []),
    "rsatb_version": (_i, []),
    "rsatb_ctx_create": (_i, [_i, C.POINTER(_vp)]),
    "rsatb_ctx_destroy": (_i, [_vp]),
    "rsatb_ctx_set_stream": (_i, [_vp, _vp]),
    "rsatb_ctx_stream": (_vp, [_vp]),
    "rsatb_ctx_synchronize": (_i, [_vp]),
    "rsatb_ctx_launch_count": (_i64, [_vp]),
    "rsatb_device_alloc": (_i, [_vp, _sz, C.POINTER(_vp)]),
    "rsatb_device_free": (_i, [_vp, _vp]),
    "rsatb_copy_to_device": (_i, [_vp, _vp, _vp, _sz]),
    "rsatb_copy_to_host_sync": (_i, [_vp, _vp, _vp, _sz]),
    "rsatb_bsr_create": (_i, [_vp, _i, _i, _i, _i64, _vp, _vp, _vp, _i, _u, C.POINTER(_vp)]),
    "rsatb_bsr_destroy": (_i, [_vp]),
    "rsatb_bsr_adjoint": (_i, [_vp, _vp, C.POINTER(_vp)]),
    "rsatb_bsr_convert": (_i, [_vp, _vp, _i, C.POINTER(_vp)]),
    "rsatb_bsr_info": (_i, [_vp, C.POINTER(_i), C.POINTER(_i), C.POINTER(_i),
                            C.POINTER(_i64), C.POINTER(_i), C.POINTER(_u)]),
    "rsatb_bsr_values": (_vp, [_vp]),
    "rsatb_bsr_pattern": (_i, [_vp, _vp, _vp, _vp]),
    "rsatb_bsr_set_values": (_i, [_vp, _vp, _vp, _u]),
    "rsatb_bsr_mult_dense": (_i, [_vp, _vp, _vp, _vp, _i, _i, _d]),
    "rsatb_cheb_apply_op": (_i, [_vp, C.POINTER(ChebOp), _vp, _vp, _i, _i]),
    "rsatb_cheb_apply_dual": (_i, [_vp, C.POINTER(ChebOp), _vp, _vp, _vp, _i, _i, _d]),
    "rsatb_cheb_apply_dual_adjoint": (_i, [_vp, C.POINTER(ChebOp), _vp, _vp, _vp, _i, _i, _d]),
    "rsatb_cheb_propagate": (_i, [_vp, C.POINTER(ChebOp), _vp, _vp, _i, _i, _PD, _i]),
    "rsatb_kpm_dos_moments": (_i, [_vp, C.POINTER(ChebOp), _vp, _i, _i, _i, _i, _PD, _PD]),
    "rsatb_kpm_dos_moments_noalloc": (_i, [_vp, C.POINTER(ChebOp), _vp, _i, _i, _i, _i, _PD,
                                           _PD]),
    "rsatb_set_random": (_i, [_vp, _u64, _i, _i, _vp, _i, _i, _i64, _i, _i64, _i, _vp]),
    "rsatb_evaluate_kpm_density": (_i, [_vp, _PD, _i, _PD, _i, _d, _i, _PD]),
    "rsatb_timeprop_coeff": (_i, [_vp, _d, _d, _i, _i, _PD, C.POINTER(_i)]),
    "rsatb_corr_dos": (_i, [_vp, _PD, _i, _i, _d, _PD, _PD]),
    "rsatb_integrate_dc_spectrum": (_i, [_vp, _PD, _PD, _i, _d, _d, _PD]),
    "rsatb_bloch_sum": (_i, [_vp, _vp, _vp, _vp, _vp, _i, _vp, _PD, _i]),
    "rsatb_cg_solve": (_i, [_vp, _vp, _vp, _vp, _vp, _vp, _i, _i, _d, _i, C.POINTER(_i), _PD]),
    "rsatb_kpm_moments_vjp": (_i, [_vp, C.POINTER(ChebOp), _vp, _i, _i, _i, _PD, _i, _PD, _vp,
                                   C.POINTER(AdjointStats)]),
    "rsatb_kpm_moments_vjp_sandwich": (_i, [_vp, C.POINTER(ChebOp), _vp, _i, _i, _i, _PD, _i,
                                            _PD, _vp, _vp, C.POINTER(AdjointStats)]),
    "rsatb_dc_spectrum_fftcheb": (_i, [_vp, C.POINTER(ChebOp), _vp, _vp, _vp, _vp, _i, _i, _i,
                                       _i, _d, _i, _sz, _i, _PD, _PD,
                                       C.POINTER(FftchebStats)]),
    "rsatb_dc_spectrum_qe": (_i, [_vp, C.POINTER(ChebOp), _vp, _vp, _vp, _vp, _i, _i, _i, _d, _i,
                                  _vp, _i, _PD, _PD]),
    "rsatb_isqrt_columns_batched": (_i, [_vp, _i, _vp, _vp, _vp, _vp, _vp, _vp, _vp,
                                         C.POINTER(IsqrtOptions), _vp, C.POINTER(IsqrtStats)]),
    "rsatb_measure_fma_peak": (_i, [_vp, _i, _PD]),
    "rsatb_isqrt_autotune": (_i, [_vp, _i, _i, _vp, _i, _vp, _vp, _vp]),
    "rsatb_inverse_sqrt_refine": (_i, [_vp, _vp, _vp, C.POINTER(NsRefineOptions),
                                       C.POINTER(_vp), C.POINTER(NsRefineReport)]),
    "rsatb_lanczos_extremes": (_i, [_vp, C.POINTER(ChebOp), C.POINTER(LanczosOptions),
                                    C.POINTER(LanczosResult)]),
    "rsatb_tridiag_eigen": (_i, [_i, _PD, _PD, _PD, _PD]),
}


def lib():
    """The loaded library; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(
                f"rsatb_b200 native library not found at {LIB_PATH}; build it with "
                "`python -m rsatb_b200.build` (nvcc, sm_100a)")
        L = C.CDLL(str(LIB_PATH))
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def exported_symbols() -> list[str]:
    return list(SIGNATURES)


def check(status: int) -> None:
    if status != SUCCESS:
        msg = lib().rsatb_last_error().decode(errors="replace")
        raise RsatbError(status, msg)
