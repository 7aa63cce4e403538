"""ctypes binding of libsptrsv_b200.so (the C ABI in include/sptrsv_b200.h).

The library is loaded from this package directory.  There is no fallback:
if the shared library is missing the import fails with instructions to build
it, so nothing can silently run on a CPU path.
"""
from __future__ import annotations

import ctypes
import os
from ctypes import POINTER, c_char_p, c_double, c_int, c_longlong, c_uint64, c_ulonglong, c_void_p
from pathlib import Path

_HERE = Path(__file__).resolve().parent
LIB_PATH = _HERE / "libsptrsv_b200.so"

# ---- enums and error codes (include/sptrsv_b200.h) ----
SIMPLE, ORDER, MULTIROW, ALL = 0, 1, 2, 3
SPTRSV_OK = 0
SPTRSV_NO_ANALYSIS = -1
SPTRSV_ERR_INVALID_ARG = -2
SPTRSV_ERR_INVALID_CSR = -3
SPTRSV_ERR_CUDA = -4
SPTRSV_ERR_TIMEOUT = -5
SPTRSV_ERR_NOT_ANALYSED = -6
SPTRSV_ERR_ALLOC = -7
SPTRSV_ERR_NOT_CONVERGED = -8
SPTRSV_ERR_UNSUPPORTED = -9

VAR_SIMPLE, VAR_ORDER, VAR_MULTIROW, VAR_CLUSTER, VAR_STRIP, VAR_WAVE, VAR_BAND = 0, 1, 2, 3, 4, 5, 6
N_VARIANTS = 6


class SpMat(ctypes.Structure):
    """sp_mat_t (header/dfr_syncfree.h:14-23)."""

    _fields_ = [("nr", c_int), ("nc", c_int), ("nnz", c_int), ("ia", c_void_p), ("ja", c_void_p), ("a", c_void_p)]


class AnalysisInfo(ctypes.Structure):
    """dfr_analysis_info_t (header/dfr_syncfree.h:25-41)."""

    _fields_ = [
        ("mode", c_int),
        ("lev_ctr", c_int),
        ("nlevs", c_int),
        ("lev_size", c_void_p),
        ("warp_lev", c_void_p),
        ("n_warps", c_int),
        ("inv_iorder", c_void_p),
        ("iorder", c_void_p),
        ("ibase_row", c_void_p),
        ("ivect_size_warp", c_void_p),
        ("row_ctr", c_void_p),
    ]


class Schedule(ctypes.Structure):
    """sptrsv_schedule_t."""

    _fields_ = [("variant", c_int), ("rows_per_warp", c_int), ("block_warps", c_int), ("warps_per_sm", c_int),
                ("backoff_ns", c_int), ("ir_max_iters", c_int), ("band_levels", c_int), ("cluster_rows", c_int),
                ("partitions", c_int)]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


class HostCsr(ctypes.Structure):
    """sptrsv_host_csr_t."""

    _fields_ = [("n", c_int), ("nnz", c_int), ("rowptr", POINTER(c_int)), ("colidx", POINTER(c_int)),
                ("val", POINTER(c_double))]


# name -> (restype, argtypes)
_SIGS = {
    "allocate_memory": (c_int, [c_void_p, c_void_p, c_void_p, c_int, POINTER(SpMat), c_int]),
    "run_analysis": (c_int, [POINTER(AnalysisInfo), POINTER(SpMat)]),
    "run_solver": (None, [POINTER(SpMat), POINTER(AnalysisInfo), c_void_p, c_void_p, c_int]),
    "free_device_analysis": (None, [POINTER(SpMat), POINTER(AnalysisInfo)]),
    "multirow_analysis_base_GPU": (None, [POINTER(POINTER(AnalysisInfo)), POINTER(SpMat), c_int]),
    "csr_L_solve_simple": (None, [POINTER(SpMat), c_void_p, c_void_p, c_int, c_void_p]),
    "csr_L_solve_order": (None, [POINTER(SpMat), POINTER(AnalysisInfo), c_void_p, c_void_p, c_int, c_void_p]),
    "csr_L_solve_multirow": (None, [POINTER(SpMat), POINTER(AnalysisInfo), c_void_p, c_void_p, c_int, c_void_p]),
    "sptrsv_last_error": (c_int, []),
    "sptrsv_last_error_string": (c_char_p, []),
    "sptrsv_version": (c_char_p, []),
    "sptrsv_sync_status": (c_int, [c_void_p]),
    "sptrsv_set_wait_budget_ns": (None, [c_ulonglong]),
    "sptrsv_selftest_bounded_wait": (c_int, [c_ulonglong]),
    "sptrsv_check_csr_host": (c_int, [c_void_p, c_void_p, c_int, POINTER(c_int)]),
    "sptrsv_analysis_levels": (c_int, [POINTER(AnalysisInfo), c_void_p]),
    "sptrsv_analysis_buckets": (c_int, [POINTER(AnalysisInfo), c_void_p]),
    "sptrsv_solve_order_tile": (c_int, [POINTER(SpMat), POINTER(AnalysisInfo), c_void_p, c_void_p, c_int, c_void_p]),
    "sptrsv_plan_create": (c_int, [POINTER(SpMat), POINTER(AnalysisInfo), POINTER(c_void_p)]),
    "sptrsv_plan_destroy": (c_int, [c_void_p]),
    "sptrsv_plan_set_schedule": (c_int, [c_void_p, POINTER(Schedule)]),
    "sptrsv_plan_get_schedule": (c_int, [c_void_p, POINTER(Schedule)]),
    "sptrsv_plan_update_values": (c_int, [c_void_p, POINTER(SpMat)]),
    "sptrsv_plan_set_stream_segment": (c_int, [c_void_p, c_int]),
    "sptrsv_partition_blocks_host": (c_int, [POINTER(HostCsr), c_int, c_void_p, POINTER(c_double)]),
    "sptrsv_plan_partition_info": (c_int, [c_void_p, POINTER(c_int), POINTER(c_int), POINTER(c_longlong),
                                           POINTER(c_double), c_void_p]),
    "sptrsv_solve_f64": (c_int, [c_void_p, c_void_p, c_void_p, c_int, c_void_p]),
    "sptrsv_solve_ir": (c_int, [c_void_p, c_void_p, c_void_p, c_int, c_void_p]),
    "sptrsv_solve_f32": (c_int, [c_void_p, c_void_p, c_void_p, c_int, c_void_p]),
    "sptrsv_plan_calibrate_ir": (c_int, [c_void_p, c_void_p, c_void_p, c_int, c_double, c_int, POINTER(c_int),
                                         POINTER(c_double)]),
    "sptrsv_solve_host": (c_int, [c_void_p, c_void_p, c_void_p, c_int, c_int, c_void_p]),
    "sptrsv_residual_f64": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_int, c_void_p]),
    "sptrsv_solve_ir_noalloc": (c_int, [POINTER(SpMat), c_void_p, c_void_p, c_int, c_void_p]),
    "sptrsv_batch_create": (c_int, [c_int, POINTER(SpMat), c_void_p, POINTER(c_void_p)]),
    "sptrsv_batch_destroy": (c_int, [c_void_p]),
    "sptrsv_batch_set_partition": (c_int, [c_void_p, c_int]),
    "sptrsv_batch_partition_info": (c_int, [c_void_p, POINTER(c_int), POINTER(c_int), POINTER(c_longlong),
                                            POINTER(c_double)]),
    "sptrsv_batch_info": (c_int, [c_void_p, c_void_p, POINTER(c_int), POINTER(c_int), POINTER(c_longlong)]),
    "sptrsv_batch_set_schedule": (c_int, [c_void_p, c_int, c_int, c_int, c_int, c_int]),
    "sptrsv_batch_set_seq_width": (c_int, [c_void_p, c_double]),
    "sptrsv_batch_seq_systems": (c_int, [c_void_p, POINTER(c_int), POINTER(c_int), POINTER(c_int)]),
    "sptrsv_batch_solve": (c_int, [c_void_p, c_void_p, c_void_p, c_int, c_void_p]),
    "sptrsv_batch_solve_graph": (c_int, [c_void_p, c_void_p, c_void_p, c_int, c_void_p]),
    "sptrsv_features": (c_int, [POINTER(SpMat), POINTER(AnalysisInfo), c_void_p]),
    "sptrsv_schedule_from_class": (c_int, [c_int, POINTER(Schedule)]),
    "sptrsv_autotune": (c_int, [c_void_p, c_void_p, c_void_p, c_int, c_int, c_int, c_void_p, POINTER(c_int)]),
    "sptrsv_mlp_create": (c_int, [c_uint64, POINTER(c_void_p)]),
    "sptrsv_mlp_destroy": (c_int, [c_void_p]),
    "sptrsv_mlp_get_params": (c_int, [c_void_p, c_void_p]),
    "sptrsv_mlp_set_params": (c_int, [c_void_p, c_void_p]),
    "sptrsv_mlp_set_normalization": (c_int, [c_void_p, c_void_p, c_void_p]),
    "sptrsv_mlp_get_normalization": (c_int, [c_void_p, c_void_p, c_void_p]),
    "sptrsv_mlp_forward_host": (c_int, [c_void_p, c_void_p, c_int, c_void_p]),
    "sptrsv_mlp_gradient_host": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_int, c_void_p, c_void_p]),
    "sptrsv_mlp_train_host": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_int, c_int, c_int, ctypes.c_float,
                                      c_uint64, c_void_p]),
    "sptrsv_mlp_predict_class": (c_int, [c_void_p, c_void_p, POINTER(c_int)]),
    "sptrsv_plan_select_schedule": (c_int, [c_void_p, c_void_p, POINTER(SpMat), POINTER(AnalysisInfo),
                                            POINTER(c_int)]),
    "sptrsv_gen_banded": (c_int, [c_int, c_int, c_int, c_int, c_uint64, POINTER(HostCsr)]),
    "sptrsv_gen_grid2d": (c_int, [c_int, c_int, c_uint64, POINTER(HostCsr)]),
    "sptrsv_gen_grid3d": (c_int, [c_int, c_int, c_int, c_uint64, POINTER(HostCsr)]),
    "sptrsv_gen_zipf": (c_int, [c_int, c_double, c_int, c_uint64, POINTER(HostCsr)]),
    "sptrsv_gen_blockdiag": (c_int, [c_int, c_int, c_uint64, POINTER(HostCsr)]),
    "sptrsv_host_csr_free": (None, [POINTER(HostCsr)]),
    "sptrsv_read_mtx_lower": (c_int, [c_char_p, c_int, POINTER(HostCsr)]),
    "sptrsv_gen_vector": (c_int, [c_longlong, c_int, c_uint64, c_void_p]),
    "sptrsv_host_spmv": (c_int, [POINTER(HostCsr), c_void_p, c_void_p, c_int]),
}

_lib = None


def lib() -> ctypes.CDLL:
    """The loaded native library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `python -m sptrsv_b200.build` "
                "(or __graft_entry__.build()); there is no CPU fallback")
        L = ctypes.CDLL(str(LIB_PATH))
        for name, (res, args) in _SIGS.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def exported_symbols():
    return list(_SIGS)


class SptrsvError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"sptrsv error {code}: {msg}")
        self.code = code


def last_error():
    L = lib()
    return L.sptrsv_last_error(), L.sptrsv_last_error_string().decode()


def check(code: int) -> int:
    """Raise SptrsvError for a negative return code."""
    if code < 0:
        _, msg = last_error()
        raise SptrsvError(code, msg)
    return code


def check_last():
    code, msg = last_error()
    if code < 0:
        raise SptrsvError(code, msg)


def default_stream():
    return None


def ptr(a) -> int:
    """Raw address of a numpy array or torch tensor."""
    if hasattr(a, "data_ptr"):
        return a.data_ptr()
    return a.ctypes.data


os.environ.setdefault("CUDA_MODULE_LOADING", "LAZY")
