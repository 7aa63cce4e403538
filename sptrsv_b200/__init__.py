"""sptrsv_b200 — B200-native sparse lower-triangular solver (SpTRSV).

A drop-in for the CSR SpTRSV path of HCL-Fing/SPTRSV: the native library
libsptrsv_b200.so (hand-written sm_100a CUDA kernels behind the C ABI in
include/sptrsv_b200.h) plus this Python mirror of the reference interface.
"""
from . import _lib
from ._lib import ALL, MULTIROW, ORDER, SIMPLE, SptrsvError, lib
from .interface import (
    AnalysisInfo,
    Plan,
    Schedule,
    SpMat,
    allocate_memory,
    analysis_arrays,
    check_csr_host,
    csr_L_solve_multirow,
    csr_L_solve_order,
    csr_L_solve_order_tile,
    csr_L_solve_simple,
    free_device_analysis,
    multirow_analysis_base_GPU,
    run_analysis,
    run_solver,
    set_wait_budget_ns,
    sync_status,
)

__all__ = [
    "SIMPLE", "ORDER", "MULTIROW", "ALL", "SptrsvError", "lib", "AnalysisInfo", "Plan", "Schedule", "SpMat",
    "allocate_memory", "analysis_arrays", "check_csr_host", "csr_L_solve_multirow", "csr_L_solve_order",
    "csr_L_solve_order_tile", "csr_L_solve_simple", "free_device_analysis", "multirow_analysis_base_GPU",
    "run_analysis", "run_solver", "set_wait_budget_ns", "sync_status",
]
