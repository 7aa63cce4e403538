"""Python mirror of the reference's CSR SpTRSV interface.

Same names, argument meaning and error behaviour as the reference's
header/interface.h:6-9, header/analysis.h:20 and header/solver.h:5-7, over
the C ABI of libsptrsv_b200.so.  Functions the reference declares as
returning int return the same codes; errors that the C ABI records as its
thread-local last error are raised as SptrsvError.

Host arrays are numpy arrays.  Device arrays (the b and x of the
csr_L_solve_* functions and of the plan solves) are torch CUDA tensors; torch
is only the device-memory and stream plumbing here.
"""
from __future__ import annotations

import ctypes
from ctypes import byref, c_int, c_void_p

import numpy as np

from . import _lib as C
from ._lib import ALL, MULTIROW, ORDER, SIMPLE, AnalysisInfo, Schedule, SpMat, SptrsvError

__all__ = [
    "SIMPLE", "ORDER", "MULTIROW", "ALL", "SpMat", "AnalysisInfo", "Schedule", "SptrsvError",
    "allocate_memory", "run_analysis", "run_solver", "free_device_analysis", "multirow_analysis_base_GPU",
    "csr_L_solve_simple", "csr_L_solve_order", "csr_L_solve_multirow", "csr_L_solve_order_tile",
    "analysis_arrays", "sync_status", "Plan", "check_csr_host", "set_wait_budget_ns",
]


def _stream(stream) -> int | None:
    if stream is None:
        return None
    if hasattr(stream, "cuda_stream"):
        return stream.cuda_stream
    return int(stream)


def _dev(t, dtype_name: str, count: int):
    if not (hasattr(t, "is_cuda") and t.is_cuda):
        raise TypeError("expected a CUDA tensor")
    if str(t.dtype) != f"torch.{dtype_name}" or not t.is_contiguous() or t.numel() < count:
        raise TypeError(f"expected a contiguous torch.{dtype_name} CUDA tensor with >= {count} elements")
    return t.data_ptr()


# ---------------------------------------------------------------- interface.h
def allocate_memory(csrRowPtrL, csrColIdxL, csrValL, n: int, mode: int = ALL) -> SpMat:
    """header/interface.h:6 — copy a host CSR to the device, return sp_mat_t."""
    rp = np.ascontiguousarray(csrRowPtrL, dtype=np.int32)
    ci = np.ascontiguousarray(csrColIdxL, dtype=np.int32)
    va = np.ascontiguousarray(csrValL, dtype=np.float64)
    if rp.shape[0] != n + 1:
        raise ValueError("csrRowPtrL must have n+1 entries")
    m = SpMat()
    C.check(C.lib().allocate_memory(rp.ctypes.data, ci.ctypes.data, va.ctypes.data, int(n), byref(m), int(mode)))
    return m


def run_analysis(info: AnalysisInfo, gpu_L: SpMat) -> int:
    """header/interface.h:7 — 0 on success, -1 for SIMPLE (interface.cu:29);
    other failures raise SptrsvError."""
    r = C.lib().run_analysis(byref(info), byref(gpu_L))
    if r == C.SPTRSV_NO_ANALYSIS:
        return r
    return C.check(r)


def run_solver(gpu_L: SpMat, info: AnalysisInfo | None, b, x, n: int) -> None:
    """header/interface.h:8 — host b in, host x out (filled in place)."""
    bb = np.ascontiguousarray(b, dtype=np.float64)
    if not (isinstance(x, np.ndarray) and x.dtype == np.float64 and x.flags.c_contiguous and x.size >= n):
        raise TypeError("x must be a contiguous float64 numpy array of n values")
    C.lib().run_solver(byref(gpu_L), byref(info) if info is not None else None, bb.ctypes.data, x.ctypes.data, int(n))
    C.check_last()


def free_device_analysis(gpu_L: SpMat | None, info: AnalysisInfo | None) -> None:
    """header/interface.h:9 — free all device arrays of both structs."""
    C.lib().free_device_analysis(byref(gpu_L) if gpu_L is not None else None,
                                 byref(info) if info is not None else None)


# ----------------------------------------------------------------- analysis.h
def multirow_analysis_base_GPU(info: AnalysisInfo, gpu_L: SpMat, mode: int) -> None:
    """header/analysis.h:20 — fills the caller-allocated info."""
    p = ctypes.pointer(info)
    C.lib().multirow_analysis_base_GPU(byref(p), byref(gpu_L), int(mode))
    C.check_last()


# ------------------------------------------------------------------- solver.h
def csr_L_solve_simple(gpu_L: SpMat, b, x, n: int, is_solved=None) -> None:
    """header/solver.h:5 — device b, x (torch float64 CUDA tensors)."""
    C.lib().csr_L_solve_simple(byref(gpu_L), _dev(b, "float64", n), _dev(x, "float64", n), int(n),
                               is_solved.data_ptr() if is_solved is not None else None)
    C.check_last()


def csr_L_solve_order(gpu_L: SpMat, info: AnalysisInfo, b, x, n: int, stream=None) -> None:
    """header/solver.h:6."""
    C.lib().csr_L_solve_order(byref(gpu_L), byref(info), _dev(b, "float64", n), _dev(x, "float64", n), int(n),
                              _stream(stream))
    C.check_last()


def csr_L_solve_multirow(gpu_L: SpMat, info: AnalysisInfo, b, x, n: int, stream=None) -> None:
    """header/solver.h:7."""
    C.lib().csr_L_solve_multirow(byref(gpu_L), byref(info), _dev(b, "float64", n), _dev(x, "float64", n), int(n),
                                 _stream(stream))
    C.check_last()


def csr_L_solve_order_tile(gpu_L: SpMat, info: AnalysisInfo, b, x, tile: int, stream=None) -> None:
    """Order with `tile` lanes per row (the reference's disabled order_coop)."""
    n = gpu_L.nr
    C.check(C.lib().sptrsv_solve_order_tile(byref(gpu_L), byref(info), _dev(b, "float64", n),
                                            _dev(x, "float64", n), int(tile), _stream(stream)))


def sync_status(stream=None) -> None:
    """Wait for the stream and raise if a bounded device wait ran out."""
    C.check(C.lib().sptrsv_sync_status(_stream(stream)))


def set_wait_budget_ns(ns: int) -> None:
    C.lib().sptrsv_set_wait_budget_ns(int(ns))


def check_csr_host(rowptr, colidx) -> int:
    """-1 if the host CSR is valid, else the first bad row."""
    rp = np.ascontiguousarray(rowptr, dtype=np.int32)
    ci = np.ascontiguousarray(colidx, dtype=np.int32)
    bad = c_int(-1)
    r = C.lib().sptrsv_check_csr_host(rp.ctypes.data, ci.ctypes.data, rp.shape[0] - 1, byref(bad))
    return -1 if r == 0 else bad.value


def _d2h(dev_ptr, count: int, dtype=np.int32) -> np.ndarray:
    out = np.empty(count, dtype=dtype)
    if count and dev_ptr:
        import torch  # noqa: F401  (ensures the CUDA runtime is initialised)
        cudart = ctypes.CDLL("libcudart.so.12")
        cudart.cudaMemcpy.argtypes = [c_void_p, c_void_p, ctypes.c_size_t, c_int]
        e = cudart.cudaMemcpy(out.ctypes.data, dev_ptr, out.nbytes, 2)
        if e != 0:
            raise RuntimeError(f"cudaMemcpy failed ({e})")
    return out


def analysis_arrays(info: AnalysisInfo, n: int) -> dict:
    """Host copies of everything an analysis produced (for tests/diagnostics)."""
    L = C.lib()
    out = {"nlevs": info.nlevs, "n_warps": info.n_warps, "mode": info.mode}
    out["iorder"] = _d2h(info.iorder, n)
    out["inv_iorder"] = _d2h(info.inv_iorder, n)
    out["lev_size"] = _d2h(info.lev_size, info.nlevs)
    if info.ibase_row:
        out["ibase_row"] = _d2h(info.ibase_row, info.n_warps + 1)
        out["ivect_size_warp"] = _d2h(info.ivect_size_warp, info.n_warps)
        out["warp_lev"] = _d2h(info.warp_lev, info.n_warps)
    lev = np.empty(max(n, 1), dtype=np.int32)
    C.check(L.sptrsv_analysis_levels(byref(info), lev.ctypes.data))
    out["levels"] = lev[:n]
    bk = np.empty(max(7 * info.nlevs, 1), dtype=np.int32)
    C.check(L.sptrsv_analysis_buckets(byref(info), bk.ctypes.data))
    out["buckets"] = bk[: 7 * info.nlevs]
    return out


# ----------------------------------------------------------------------- plan
class Plan:
    """Solve plan over an analysed matrix (level-ordered copy of L)."""

    def __init__(self, gpu_L: SpMat, info: AnalysisInfo):
        h = c_void_p()
        C.check(C.lib().sptrsv_plan_create(byref(gpu_L), byref(info), byref(h)))
        self._h = h
        self.n = gpu_L.nr

    @property
    def handle(self):
        return self._h

    def set_schedule(self, variant: int, rows_per_warp: int = 1, ir_max_iters: int = 2, block_warps: int = 8,
                     warps_per_sm: int = 0, backoff_ns: int = 0, band_levels: int = 64, cluster_rows: int = 4096,
                     partitions: int = 0):
        s = Schedule(variant, rows_per_warp, block_warps, warps_per_sm, backoff_ns, ir_max_iters, band_levels,
                     cluster_rows, partitions)
        C.check(C.lib().sptrsv_plan_set_schedule(self._h, byref(s)))

    def set_schedule_struct(self, s: Schedule):
        C.check(C.lib().sptrsv_plan_set_schedule(self._h, byref(s)))

    def schedule(self) -> Schedule:
        s = Schedule()
        C.check(C.lib().sptrsv_plan_get_schedule(self._h, byref(s)))
        return s

    def update_values(self, gpu_L: SpMat):
        C.check(C.lib().sptrsv_plan_update_values(self._h, byref(gpu_L)))

    def set_stream_segment(self, rows: int):
        """Rows per copied segment of b in streamed host solves (0: default)."""
        C.check(C.lib().sptrsv_plan_set_stream_segment(self._h, int(rows)))

    def partition_info(self) -> dict:
        """Blocks of a partitioned schedule: count, block-system rows, warm-up
        rows, truncation bound and the (s, a, e, base) table per block."""
        nb, ne, wr, bd = C.c_int(), C.c_int(), C.c_longlong(), C.c_double()
        C.check(C.lib().sptrsv_plan_partition_info(self._h, byref(nb), byref(ne), byref(wr), byref(bd), None))
        tab = np.zeros(4 * nb.value, dtype=np.int32)
        C.check(C.lib().sptrsv_plan_partition_info(self._h, None, None, None, None, tab.ctypes.data))
        return {"blocks": nb.value, "n_ext": ne.value, "warm_rows": wr.value, "bound": bd.value,
                "table": tab.reshape(-1, 4)}

    def solve_f64(self, b, x, nrhs: int = 1, stream=None):
        m = self.n * nrhs
        C.check(C.lib().sptrsv_solve_f64(self._h, _dev(b, "float64", m), _dev(x, "float64", m), nrhs, _stream(stream)))

    def solve_ir(self, b, x, nrhs: int = 1, stream=None):
        m = self.n * nrhs
        C.check(C.lib().sptrsv_solve_ir(self._h, _dev(b, "float64", m), _dev(x, "float64", m), nrhs, _stream(stream)))

    def calibrate_ir(self, b, x, nrhs: int = 1, tol: float = 1e-13, max_iters: int = 4):
        """Sets and returns the refinement step count for this plan."""
        m = self.n * nrhs
        it, est = c_int(0), ctypes.c_double(0)
        C.check(C.lib().sptrsv_plan_calibrate_ir(self._h, _dev(b, "float64", m), _dev(x, "float64", m), nrhs, tol,
                                                 max_iters, byref(it), byref(est)))
        return it.value, est.value

    def solve_f32(self, b, x32, nrhs: int = 1, stream=None):
        m = self.n * nrhs
        C.check(C.lib().sptrsv_solve_f32(self._h, _dev(b, "float64", m), _dev(x32, "float32", m), nrhs,
                                         _stream(stream)))

    def residual(self, b, x, r, nrhs: int = 1, stream=None):
        m = self.n * nrhs
        C.check(C.lib().sptrsv_residual_f64(self._h, _dev(b, "float64", m), _dev(x, "float64", m),
                                            _dev(r, "float64", m), nrhs, _stream(stream)))

    def solve_host(self, b: np.ndarray, x: np.ndarray, nrhs: int = 1, precision: int = 32, stream=None):
        """Host b in, host x out; copies happen on `stream` inside the call."""
        m = self.n * nrhs
        for a in (b, x):
            size = a.numel() if hasattr(a, "numel") else a.size
            if "float64" not in str(a.dtype) or size < m or getattr(a, "is_cuda", False):
                raise TypeError("b and x must be host float64 arrays of n*nrhs values")
        C.check(C.lib().sptrsv_solve_host(self._h, C.ptr(b), C.ptr(x), nrhs, precision, _stream(stream)))

    def close(self):
        if self._h:
            C.lib().sptrsv_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
