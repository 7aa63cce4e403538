"""ctypes binding of the CPU oracle (oracle/liboracle.so) and of the
reference's own kernels built from source (oracle/_ref/libsptrsv_ref.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py, as the checker or the timed CPU baseline.  The
library (sptrsv_b200) never imports it.
"""
from __future__ import annotations

import ctypes
import subprocess
import time
from ctypes import POINTER, c_double, c_float, c_int, c_size_t, c_void_p
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ORACLE_SO = HERE / "liboracle.so"
REF_SO = HERE / "_ref" / "libsptrsv_ref.so"

_o = None
_r = None


def build_oracle() -> Path:
    if not ORACLE_SO.exists() or ORACLE_SO.stat().st_mtime < (HERE / "sptrsv_oracle.c").stat().st_mtime:
        subprocess.run(["make", "-s", "-C", str(HERE), "liboracle.so"], check=True)
    return ORACLE_SO


def lib():
    global _o
    if _o is None:
        build_oracle()
        L = ctypes.CDLL(str(ORACLE_SO))
        L.oracle_levels.restype = c_int
        L.oracle_levels.argtypes = [c_int, c_void_p, c_void_p, c_void_p]
        L.oracle_bucket.restype = c_int
        L.oracle_bucket.argtypes = [c_int]
        L.oracle_order.restype = None
        L.oracle_order.argtypes = [c_int, c_void_p, c_void_p, c_int, c_void_p, c_void_p]
        L.oracle_n_warps.restype = c_int
        L.oracle_n_warps.argtypes = [c_int, c_void_p]
        L.oracle_warp_map.restype = None
        L.oracle_warp_map.argtypes = [c_int, c_int, c_void_p, c_void_p, c_void_p, c_void_p]
        for f in ("oracle_solve_f64", "oracle_solve_ld", "oracle_solve_f32", "oracle_spmv"):
            getattr(L, f).restype = None
            getattr(L, f).argtypes = [c_int, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_int]
        L.oracle_solve_levels_omp.restype = None
        L.oracle_solve_levels_omp.argtypes = [c_int, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_int,
                                              c_void_p, c_void_p, c_int]
        L.oracle_num_threads.restype = c_int
        L.oracle_rel_err_inf.restype = c_double
        L.oracle_rel_err_inf.argtypes = [c_size_t, c_void_p, c_void_p]
        L.mlp_oracle_nparams.restype = c_int
        L.mlp_oracle_forward.restype = None
        L.mlp_oracle_forward.argtypes = [c_void_p, c_void_p, c_void_p, c_void_p, c_int, c_void_p]
        L.mlp_oracle_gradient.restype = c_double
        L.mlp_oracle_gradient.argtypes = [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_int,
                                          c_void_p]
        _o = L
    return _o


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def analysis(rowptr, colidx) -> dict:
    """Levels, nlevs, iorder, buckets and the multirow warp map
    (analysis/analysis_csr.cu:104-410 restated)."""
    L = lib()
    rp, ci = _i32(rowptr), _i32(colidx)
    n = rp.shape[0] - 1
    lev = np.zeros(max(n, 1), dtype=np.int32)
    nlevs = L.oracle_levels(n, rp.ctypes.data, ci.ctypes.data, lev.ctypes.data)
    iorder = np.zeros(max(n, 1), dtype=np.int32)
    buckets = np.zeros(7 * nlevs + 1, dtype=np.int32)
    L.oracle_order(n, rp.ctypes.data, lev.ctypes.data, nlevs, iorder.ctypes.data, buckets.ctypes.data)
    nw = L.oracle_n_warps(nlevs, buckets.ctypes.data)
    ibase = np.zeros(nw + 1, dtype=np.int32)
    ivect = np.zeros(max(nw, 1), dtype=np.int32)
    wlev = np.zeros(max(nw, 1), dtype=np.int32)
    L.oracle_warp_map(n, nlevs, buckets.ctypes.data, ibase.ctypes.data, ivect.ctypes.data, wlev.ctypes.data)
    return {"levels": lev[:n], "nlevs": nlevs, "iorder": iorder[:n], "buckets": buckets[: 7 * nlevs],
            "n_warps": nw, "ibase_row": ibase, "ivect_size_warp": ivect[:nw], "warp_lev": wlev[:nw]}


def solve(rowptr, colidx, val, b, nrhs: int = 1, long_double: bool = False, f32: bool = False) -> np.ndarray:
    """Serial substitution: FP64 (default), long double, or the reference's
    FP32 build restated in float (f32)."""
    L = lib()
    rp, ci, va, bb = _i32(rowptr), _i32(colidx), _f64(val), _f64(b)
    n = rp.shape[0] - 1
    x = np.zeros(max(n * nrhs, 1), dtype=np.float64)
    f = L.oracle_solve_ld if long_double else L.oracle_solve_f32 if f32 else L.oracle_solve_f64
    f(n, rp.ctypes.data, ci.ctypes.data, va.ctypes.data, bb.ctypes.data, x.ctypes.data, nrhs)
    return x[: n * nrhs]


def solve_levels_omp(rowptr, colidx, val, b, iorder, lev_ptr, nlevs, nrhs=1) -> np.ndarray:
    L = lib()
    rp, ci, va, bb = _i32(rowptr), _i32(colidx), _f64(val), _f64(b)
    io, lp = _i32(iorder), _i32(lev_ptr)
    n = rp.shape[0] - 1
    x = np.zeros(max(n * nrhs, 1), dtype=np.float64)
    L.oracle_solve_levels_omp(n, rp.ctypes.data, ci.ctypes.data, va.ctypes.data, io.ctypes.data, lp.ctypes.data,
                              nlevs, bb.ctypes.data, x.ctypes.data, nrhs)
    return x[: n * nrhs]


def spmv(rowptr, colidx, val, x, nrhs: int = 1) -> np.ndarray:
    L = lib()
    rp, ci, va, xx = _i32(rowptr), _i32(colidx), _f64(val), _f64(x)
    n = rp.shape[0] - 1
    y = np.zeros(max(n * nrhs, 1), dtype=np.float64)
    L.oracle_spmv(n, rp.ctypes.data, ci.ctypes.data, va.ctypes.data, xx.ctypes.data, y.ctypes.data, nrhs)
    return y[: n * nrhs]


def rel_err(a, b) -> float:
    a, b = _f64(a), _f64(b)
    return lib().oracle_rel_err_inf(a.size, a.ctypes.data, b.ctypes.data)


def num_threads() -> int:
    return lib().oracle_num_threads()


# ---- MLP oracle (oracle/mlp_oracle.c) ----
def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def mlp_forward(params, mean, std, X) -> np.ndarray:
    P, m, s, Xf = _f32(params), _f32(mean), _f32(std), _f32(X).reshape(-1, 12)
    Y = np.zeros((Xf.shape[0], 24), dtype=np.float64)
    lib().mlp_oracle_forward(P.ctypes.data, m.ctypes.data, s.ctypes.data, Xf.ctypes.data, Xf.shape[0], Y.ctypes.data)
    return Y


def mlp_gradient(params, mean, std, X, T, M):
    P, m, s = _f32(params), _f32(mean), _f32(std)
    Xf, Tf, Mf = _f32(X).reshape(-1, 12), _f32(T).reshape(-1, 24), _f32(M).reshape(-1, 24)
    G = np.zeros(lib().mlp_oracle_nparams(), dtype=np.float64)
    loss = lib().mlp_oracle_gradient(P.ctypes.data, m.ctypes.data, s.ctypes.data, Xf.ctypes.data, Tf.ctypes.data,
                                     Mf.ctypes.data, Xf.shape[0], G.ctypes.data)
    return loss, G


# ---- the reference's own kernels (GPU only; built by `make -C oracle ref`) ----
def ref_available() -> bool:
    return REF_SO.exists()


def ref_lib():
    """The reference's FP64 kernels built from its sources (oracle/_ref)."""
    global _r
    if _r is None:
        if not REF_SO.exists():
            raise FileNotFoundError(f"{REF_SO} not built (make -C oracle ref, needs the reference sources)")
        _r = _bind_ref(ctypes.CDLL(str(REF_SO)))
    return _r


def _bind_ref(L):
    L.ref_analysis.restype = c_int
    L.ref_analysis.argtypes = [c_int, c_void_p, c_void_p, c_int, POINTER(c_int), POINTER(c_int), c_void_p,
                               c_void_p, c_void_p, c_void_p]
    L.ref_solve.restype = c_int
    L.ref_solve.argtypes = [c_int, c_int, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_int,
                            POINTER(c_float)]
    L.ref_set_watchdog_seconds.restype = None
    L.ref_set_watchdog_seconds.argtypes = [c_double]
    return L


def ref_analysis(rowptr, colidx, mode: int = 2) -> dict:
    """The reference's multirow_analysis_base_GPU on a B200 (mode 1 ORDER, 2 MULTIROW)."""
    L = ref_lib()
    rp, ci = _i32(rowptr), _i32(colidx)
    n = rp.shape[0] - 1
    nlevs, nw = c_int(0), c_int(0)
    lev = np.zeros(n, dtype=np.int32)
    io = np.zeros(n, dtype=np.int32)
    ib = np.zeros(n + 1, dtype=np.int32)
    iv = np.zeros(n, dtype=np.int32)
    rc = L.ref_analysis(n, rp.ctypes.data, ci.ctypes.data, mode, ctypes.byref(nlevs), ctypes.byref(nw),
                        lev.ctypes.data, io.ctypes.data, ib.ctypes.data, iv.ctypes.data)
    if rc != 0:
        raise RuntimeError(f"ref_analysis failed ({rc})")
    w = nw.value
    out = {"levels": lev, "nlevs": nlevs.value, "iorder": io}
    if mode in (2, 3):
        out.update({"n_warps": w, "ibase_row": ib[: w + 1], "ivect_size_warp": iv[:w]})
    return out


def ref_solve(variant: int, rowptr, colidx, val, b, reps: int = 1):
    """(x, median ms) of the reference solver 0 simple, 1 order, 2 multirow."""
    L = ref_lib()
    rp, ci, va, bb = _i32(rowptr), _i32(colidx), _f64(val), _f64(b)
    n = rp.shape[0] - 1
    x = np.zeros(n, dtype=np.float64)
    ms = c_float(0)
    rc = L.ref_solve(variant, n, rp.ctypes.data, ci.ctypes.data, va.ctypes.data, bb.ctypes.data, x.ctypes.data,
                     reps, ctypes.byref(ms))
    if rc != 0:
        raise RuntimeError(f"ref_solve failed ({rc})")
    return x, ms.value


CUSPARSE_SO = HERE / "libcusparse_cmp.so"


def cusparse_solve(rowptr, colidx, val, b, reps: int = 5):
    """(x, solve ms, analysis ms) of cusparseSpSV (FP64), the comparator the
    reference's csrsv2 wrapper (solver/solve_csr_cusparse.cu) maps to."""
    if not CUSPARSE_SO.exists():
        subprocess.run(["make", "-s", "-C", str(HERE), "libcusparse_cmp.so"], check=True)
    L = ctypes.CDLL(str(CUSPARSE_SO))
    L.cmp_cusparse_spsv.restype = c_int
    L.cmp_cusparse_spsv.argtypes = [c_int, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_int,
                                    POINTER(c_float), POINTER(c_float)]
    rp, ci, va, bb = _i32(rowptr), _i32(colidx), _f64(val), _f64(b)
    n = rp.shape[0] - 1
    x = np.zeros(n)
    sm, am = c_float(0), c_float(0)
    rc = L.cmp_cusparse_spsv(n, rp.ctypes.data, ci.ctypes.data, va.ctypes.data, bb.ctypes.data, x.ctypes.data, reps,
                             ctypes.byref(sm), ctypes.byref(am))
    if rc != 0:
        raise RuntimeError(f"cusparse comparator failed ({rc})")
    return x, sm.value, am.value


def timed(fn, *a, **k):
    t0 = time.perf_counter()
    r = fn(*a, **k)
    return r, time.perf_counter() - t0
