"""thermofem_b200 -- B200 (sm_100a) sparse solve path of ThermoFEM.

Python binding of the C ABI in include/thermofem_b200.h (ctypes over
thermofem_b200/lib/libthermofem_b200.so).  Device memory comes from torch
tensors; every computation runs in the CUDA library.  There is no CPU path:
importing works without a GPU (so the C ABI can be inspected), but every
compute call needs a CUDA device and raises otherwise.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "lib", "libthermofem_b200.so")

OK, ERR_INVALID, ERR_CUDA, ERR_LENGTH, ERR_LOGIC, ERR_TIMEOUT, ERR_NOMEM, ERR_RUNTIME = 0, -1, -2, -3, -4, -5, -6, -7
F32, F64, I32, I64 = 0, 1, 2, 3
F32_VALUES = 4  # tf_amg_options.hierarchy_type: FP32 operators under an FP64 cycle
CYCLE = {"v": 0, "w": 1, "f": 2}
SOLVER_CG, SOLVER_BICGSTAB = 0, 1
PRECOND_IDENTITY, PRECOND_AMG = 0, 1
STATUS = ["Converged", "MaxIterations", "Breakdown", "NonFinite"]


class ThermoError(RuntimeError):
    """Base class of errors reported by the C ABI."""

    def __init__(self, status: int, message: str):
        super().__init__(message)
        self.status = status


class InvalidArgument(ThermoError, ValueError):
    """TF_ERR_INVALID (std::invalid_argument in the reference)."""


class LengthError(ThermoError, ValueError):
    """TF_ERR_LENGTH (std::length_error)."""


class LogicError(ThermoError):
    """TF_ERR_LOGIC (std::logic_error, e.g. apply before setup)."""


class CudaError(ThermoError):
    """TF_ERR_CUDA / TF_ERR_NOMEM."""


class TimeoutError_(ThermoError):
    """TF_ERR_TIMEOUT: a bounded device wait gave up."""


class ParseError(ThermoError):
    """TF_ERR_RUNTIME (std::runtime_error, e.g. malformed Matrix Market)."""


_ERRORS = {ERR_INVALID: InvalidArgument, ERR_LENGTH: LengthError, ERR_LOGIC: LogicError, ERR_CUDA: CudaError,
           ERR_NOMEM: CudaError, ERR_TIMEOUT: TimeoutError_, ERR_RUNTIME: ParseError}


class Csr(C.Structure):
    """tf_csr: device CSR view."""
    _fields_ = [("rows", C.c_int64), ("cols", C.c_int64), ("nnz", C.c_int64), ("index_type", C.c_int),
                ("value_type", C.c_int), ("offsets", C.c_void_p), ("indices", C.c_void_p), ("values", C.c_void_p)]


class AmgOptions(C.Structure):
    """tf_amg_options (AmgOptions of include/Preconditioner/Amg.cuh plus precision)."""
    _fields_ = [("max_levels", C.c_int), ("coarse_rows", C.c_int), ("matching_rounds", C.c_int),
                ("pre_sweeps", C.c_int), ("post_sweeps", C.c_int), ("coarse_sweeps", C.c_int),
                ("jacobi_weight", C.c_double), ("strength_threshold", C.c_double),
                ("absorb_singletons", C.c_int), ("compact_sort_keys", C.c_int), ("cycle", C.c_int),
                ("hierarchy_type", C.c_int), ("coarse_lu_rows", C.c_int), ("small_level_rows", C.c_int),
                ("damping_model", C.c_void_p)]


class SolverOptions(C.Structure):
    _fields_ = [("max_iterations", C.c_int), ("relative_tolerance", C.c_double),
                ("absolute_tolerance", C.c_double), ("residual_refresh_interval", C.c_int)]


class SolveResult(C.Structure):
    _fields_ = [("status", C.c_int), ("iterations", C.c_int), ("residual_norm", C.c_double),
                ("relative_residual", C.c_double)]

    def as_dict(self):
        return {"status": STATUS[self.status], "iterations": self.iterations,
                "residual_norm": self.residual_norm, "relative_residual": self.relative_residual}


class HostCsr(C.Structure):
    _fields_ = [("rows", C.c_int), ("cols", C.c_int), ("nnz", C.c_int64), ("offsets", C.POINTER(C.c_int32)),
                ("indices", C.POINTER(C.c_int32)), ("values", C.POINTER(C.c_double))]


# The byte source of tf_read_matrix_market_stream: read(user, buf, capacity).
MM_READ = C.CFUNCTYPE(C.c_size_t, C.c_void_p, C.c_void_p, C.c_size_t)

# Every symbol declared in include/thermofem_b200.h with its ctypes signature.
_P, _I, _L, _D, _S = C.c_void_p, C.c_int, C.c_int64, C.c_double, C.c_size_t
_PP = C.POINTER(C.c_void_p)
SIGNATURES = {
    "tf_version": ([], C.c_char_p),
    "tf_last_error": ([], C.c_char_p),
    "tf_last_cuda_error": ([], _I),
    "tf_status_string": ([_I], C.c_char_p),
    "tf_ctx_create": ([_I, _P, _PP], _I),
    "tf_ctx_destroy": ([_P], _I),
    "tf_ctx_synchronize": ([_P], _I),
    "tf_ctx_check_bounded_wait": ([_P, _L], _I),
    "tf_ctx_stream": ([_P], _P),
    "tf_ctx_device": ([_P], _I),
    "tf_ctx_launch_count": ([_P], _L),
    "tf_device_count": ([C.POINTER(C.c_int)], _I),
    "tf_dcsr_view": ([_P, C.POINTER(Csr)], _I),
    "tf_dcsr_free": ([_P], _I),
    "tf_csr_validate": ([_P, C.POINTER(Csr)], _I),
    "tf_csr_check_canonical": ([_P, C.POINTER(Csr), C.POINTER(C.c_int)], _I),
    "tf_canonicalize": ([_P, C.POINTER(Csr), _PP], _I),
    "tf_convert": ([_P, _L, _I, _P, _I, _P], _I),
    "tf_spmv": ([_P, C.POINTER(Csr), _P, _P], _I),
    "tf_spmv_f64": ([_P, _L, _L, _L, _P, _P, _P, _P, _P], _I),
    "tf_spmv_f32": ([_P, _L, _L, _L, _P, _P, _P, _P, _P], _I),
    "tf_residual": ([_P, C.POINTER(Csr), _P, _P, _P], _I),
    "tf_autotune_spmv": ([_P, C.POINTER(Csr), _P, _P, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int),
                          C.POINTER(C.c_int), C.POINTER(C.c_float)], _I),
    "tf_spmv_set_config": ([_P, C.POINTER(Csr), _I, _I, _I, _I], _I),
    "tf_jacobi_sweep": ([_P, C.POINTER(Csr), _P, _P, _P, _P, _D, _P, _P, _P], _I),
    "tf_jacobi_zero": ([_P, _L, _I, _P, _P, _P, _D, _P], _I),
    "tf_jacobi_update": ([_P, _I, _L, _D, _P, _P, _P, _P], _I),
    "tf_inverse_diagonal": ([_P, C.POINTER(Csr), _P], _I),
    "tf_restrict": ([_P, _I, _L, _P, _P, _P, _P], _I),
    "tf_prolong": ([_P, _I, _L, _P, _P, _P], _I),
    "tf_dot_multi": ([_P, _I, _L, _I, _PP, _PP, _P], _I),
    "tf_axpby": ([_P, _I, _L, _D, _P, _D, _P], _I),
    "tf_krylov_cg_update": ([_P, _I, _L, _D, _P, _P, _P, _P, _P], _I),
    "tf_krylov_cg_direction": ([_P, _I, _L, _D, _I, _P, _P], _I),
    "tf_krylov_bicgstab_direction": ([_P, _I, _L, _D, _D, _I, _P, _P, _P], _I),
    "tf_krylov_bicgstab_s": ([_P, _I, _L, _D, _P, _P, _P, _P, _P, _P], _I),
    "tf_krylov_bicgstab_update": ([_P, _I, _L, _D, _P, _P, _P, _P, _P, _P], _I),
    "tf_row_stats": ([_P, C.POINTER(Csr), _P, C.POINTER(C.c_int)], _I),
    "tf_strength": ([_P, C.POINTER(Csr), _P, _D, _PP], _I),
    "tf_match": ([_P, C.POINTER(Csr), _I, _P, C.POINTER(C.c_int)], _I),
    "tf_contract": ([_P, C.POINTER(Csr), _P, _I, _PP], _I),
    "tf_aggregate": ([_P, C.POINTER(Csr), _I, _I, _PP], _I),
    "tf_transfer_info": ([_P, C.POINTER(C.c_int), C.POINTER(C.c_int), _P], _I),
    "tf_transfer_arrays": ([_P, _PP, _PP, _PP], _I),
    "tf_transfer_free": ([_P], _I),
    "tf_galerkin": ([_P, C.POINTER(Csr), _P, _PP], _I),
    "tf_galerkin_map": ([_P, C.POINTER(Csr), _P, _I, _PP], _I),
    "tf_radix_sort_pairs_u64f64": ([_P, _L, _P, _P, _P, _P, _I], _I),
    "tf_reduce_by_key_u64f64": ([_P, _L, _P, _P, _I, _P, _P, C.POINTER(C.c_int64)], _I),
    "tf_scan_exclusive_i32": ([_P, _L, _P, _P], _I),
    "tf_scan_exclusive_i32_noalloc": ([_P, _L, _P, _P], _I),
    "tf_coarse_lu_factor": ([_P, C.POINTER(Csr), _P, _P, C.POINTER(C.c_int)], _I),
    "tf_coarse_lu_solve": ([_P, _I, _P, _P, _I, _P, _P], _I),
    "tf_amg_options_default": ([C.POINTER(AmgOptions)], None),
    "tf_amg_create": ([_P, _I, _I, C.POINTER(AmgOptions), _PP], _I),
    "tf_amg_destroy": ([_P], _I),
    "tf_amg_setup": ([_P, C.POINTER(Csr)], _I),
    "tf_amg_apply": ([_P, _P, _P], _I),
    "tf_amg_level_count": ([_P], _I),
    "tf_amg_level_stats": ([_P, _I, C.POINTER(C.c_int64), C.POINTER(C.c_int64), _P], _I),
    "tf_amg_stop_reason": ([_P], C.c_char_p),
    "tf_amg_coarse_solver": ([_P], C.c_char_p),
    "tf_amg_last_visits": ([_P, _P, _I], _I),
    "tf_amg_setup_phases": ([_P, _P, _I], _I),
    "tf_amg_setup_phase_count": ([], _I),
    "tf_amg_setup_phase_name": ([_I], C.c_char_p),
    "tf_amg_level_matrix": ([_P, _I, C.POINTER(Csr)], _I),
    "tf_amg_level_transfer": ([_P, _I, _PP, _PP, _PP, C.POINTER(C.c_int)], _I),
    "tf_amg_coarse_factor": ([_P, C.POINTER(C.c_int), _PP, _PP], _I),
    "tf_amg_save": ([C.c_void_p, C.c_char_p], C.c_int),
    "tf_amg_load": ([C.c_void_p, C.c_char_p], C.c_int),
    "tf_jacobi_create": ([_P, _I, _I, _I, _D, _PP], _I),
    "tf_jacobi_destroy": ([_P], _I),
    "tf_jacobi_setup": ([_P, C.POINTER(Csr)], _I),
    "tf_jacobi_apply": ([_P, _P, _P], _I),
    "tf_solver_options_default": ([_I, C.POINTER(SolverOptions)], None),
    "tf_solver_create": ([_P, _I, _I, _I, C.POINTER(SolverOptions), _I, C.POINTER(AmgOptions), _PP], _I),
    "tf_solver_destroy": ([_P], _I),
    "tf_solver_setup": ([_P, C.POINTER(Csr)], _I),
    "tf_solver_apply": ([_P, _P, _P, _I, C.POINTER(SolveResult)], _I),
    "tf_solver_amg": ([_P], _P),
    "tf_solver_set_graph_mode": ([_P, _I], _I),
    "tf_solver_last_apply_ms": ([_P], _D),
    "tf_solver_last_execution": ([_P], _I),
    "tf_solver_spmv": ([_P, _P, _P], _I),
    "tf_solver_spmv_layout": ([_P, C.POINTER(C.c_int), C.POINTER(C.c_int64)], _I),
    "tf_batch_create": ([_P, _I, _PP, _PP], _I),
    "tf_batch_destroy": ([_P], _I),
    "tf_batch_apply": ([_P, _PP, _PP, C.POINTER(SolveResult)], _I),
    "tf_amg_level_spmv": ([_P, _I, _P, _P], _I),
    "tf_amg_level_spmv_layout": ([_P, _I, C.POINTER(C.c_int), C.POINTER(C.c_int64)], _I),
    "tf_mlp_create": ([_P, C.c_uint64, _D, _D, _PP], _I),
    "tf_mlp_destroy": ([_P], _I),
    "tf_mlp_get_params": ([_P, C.POINTER(C.c_float)], _I),
    "tf_mlp_set_params": ([_P, C.POINTER(C.c_float)], _I),
    "tf_mlp_bounds": ([_P, C.POINTER(C.c_double), C.POINTER(C.c_double)], _I),
    "tf_row_features": ([_P, C.POINTER(Csr), _I, _P], _I),
    "tf_mlp_forward": ([_P, _L, _P, _P], _I),
    "tf_mlp_backward": ([_P, _L, _P, _P, C.POINTER(C.c_double)], _I),
    "tf_mlp_get_gradient": ([_P, C.POINTER(C.c_double)], _I),
    "tf_mlp_sgd": ([_P, _D, _D], _I),
    "tf_read_matrix_market": ([C.c_char_p, _S, C.POINTER(HostCsr)], _I),
    "tf_read_matrix_market_file": ([C.c_char_p, C.POINTER(HostCsr)], _I),
    "tf_read_matrix_market_stream": ([MM_READ, _P, C.POINTER(HostCsr)], _I),
    "tf_host_csr_free": ([C.POINTER(HostCsr)], None),
}

_lib = None


def lib():
    """Loads the CUDA library; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `python -m thermofem_b200.build`")
        L = C.CDLL(LIB_PATH)
        for name, (args, res) in SIGNATURES.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = res
        _lib = L
    return _lib


def check(status: int):
    if status != OK:
        msg = lib().tf_last_error().decode(errors="replace")
        raise _ERRORS.get(status, ThermoError)(status, msg or lib().tf_status_string(status).decode())


def device_count() -> int:
    n = C.c_int(0)
    check(lib().tf_device_count(C.byref(n)))
    return n.value


def version() -> str:
    return lib().tf_version().decode()


from .api import *  # noqa: E402,F401,F403
from . import api  # noqa: E402,F401
