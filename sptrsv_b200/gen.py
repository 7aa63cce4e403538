"""Seeded synthetic matrices (the benchmark configurations) as numpy CSR.

Thin wrappers over the generators in libsptrsv_b200.so (csrc/gen.cpp).
"""
from __future__ import annotations

from ctypes import byref
from dataclasses import dataclass

import numpy as np

from . import _lib as C


@dataclass
class HostCsr:
    """Lower-triangular CSR on the host: sorted columns, diagonal last."""

    rowptr: np.ndarray
    colidx: np.ndarray
    val: np.ndarray

    @property
    def n(self) -> int:
        return int(self.rowptr.shape[0] - 1)

    @property
    def nnz(self) -> int:
        return int(self.rowptr[-1])

    def matvec(self, x: np.ndarray, nrhs: int = 1) -> np.ndarray:
        """y = L x in FP64, column order per row (host)."""
        hc = C.HostCsr(self.n, self.nnz, self.rowptr.ctypes.data_as(C.POINTER(C.c_int)),
                       self.colidx.ctypes.data_as(C.POINTER(C.c_int)),
                       self.val.ctypes.data_as(C.POINTER(C.c_double)))
        xx = np.ascontiguousarray(x, dtype=np.float64)
        y = np.empty(self.n * nrhs, dtype=np.float64)
        C.check(C.lib().sptrsv_host_spmv(byref(hc), xx.ctypes.data, y.ctypes.data, nrhs))
        return y

    def unit_values(self) -> "HostCsr":
        """Same pattern with every value 1.0 (the reference's test input, main.cu:228,236)."""
        return HostCsr(self.rowptr, self.colidx, np.ones_like(self.val))


def _take(fn, *args) -> HostCsr:
    h = C.HostCsr()
    C.check(fn(*args, byref(h)))
    try:
        n, nnz = h.n, h.nnz
        rp = np.ctypeslib.as_array(h.rowptr, shape=(n + 1,)).copy()
        ci = np.ctypeslib.as_array(h.colidx, shape=(max(nnz, 1),))[:nnz].copy()
        va = np.ctypeslib.as_array(h.val, shape=(max(nnz, 1),))[:nnz].copy()
    finally:
        C.lib().sptrsv_host_csr_free(byref(h))
    return HostCsr(rp, ci, va)


def banded(n: int, bandwidth: int = 256, off_min: int = 8, off_max: int = 8, seed: int = 0) -> HostCsr:
    return _take(C.lib().sptrsv_gen_banded, n, bandwidth, off_min, off_max, seed)


def grid2d(nx: int, ny: int | None = None, seed: int = 1) -> HostCsr:
    return _take(C.lib().sptrsv_gen_grid2d, nx, ny if ny is not None else nx, seed)


def grid3d(nx: int, ny: int | None = None, nz: int | None = None, seed: int = 0) -> HostCsr:
    return _take(C.lib().sptrsv_gen_grid3d, nx, ny or nx, nz or nx, seed)


def zipf(n: int, s: float = 1.5, max_off: int = 256, seed: int = 2) -> HostCsr:
    return _take(C.lib().sptrsv_gen_zipf, n, s, max_off, seed)


def blockdiag(n: int, block: int = 32, seed: int = 0) -> HostCsr:
    return _take(C.lib().sptrsv_gen_blockdiag, n, block, seed)


def vector(m: int, dist: str = "ones", seed: int = 0) -> np.ndarray:
    """dist: 'ones', 'uniform' (U(-1,1)) or 'normal' (N(0,1))."""
    code = {"ones": 0, "uniform": 1, "normal": 2}[dist]
    out = np.empty(m, dtype=np.float64)
    C.check(C.lib().sptrsv_gen_vector(m, code, seed, out.ctypes.data))
    return out


def read_mtx_lower(path, unit_values: bool = True) -> HostCsr:
    """Lower triangle (diagonal last) of a MatrixMarket file; unit_values
    reproduces the reference driver's all-ones values."""
    return _take(C.lib().sptrsv_read_mtx_lower, str(path).encode(), 1 if unit_values else 0)


def from_arrays(rowptr, colidx, val) -> HostCsr:
    return HostCsr(np.ascontiguousarray(rowptr, np.int32), np.ascontiguousarray(colidx, np.int32),
                   np.ascontiguousarray(val, np.float64))


def batch_config(nsys: int = 512, seed: int = 3, n_lo: int = 1000, n_hi: int = 200_000, bw_lo: int = 16,
                 bw_hi: int = 4096, off_lo: int = 4, off_hi: int = 16, k_max: int = 32):
    """Batched configuration: nsys banded systems with n log-uniform in
    [n_lo, n_hi], bandwidth log-uniform in [bw_lo, bw_hi], off_lo..off_hi
    off-diagonals per row, k ~ U{1..k_max} right-hand sides each.
    Returns (list of HostCsr, list of nrhs, list of x_true (row-major n x k))."""
    rng = np.random.default_rng(seed)
    ns = np.exp(rng.uniform(np.log(n_lo), np.log(n_hi), nsys)).astype(np.int64)
    bws = np.exp(rng.uniform(np.log(bw_lo), np.log(bw_hi), nsys)).astype(np.int64)
    ks = rng.integers(1, k_max + 1, nsys)
    mats, xs = [], []
    for s in range(nsys):
        mats.append(banded(int(ns[s]), int(bws[s]), off_lo, off_hi, seed=seed * 1_000_003 + s))
        xs.append(vector(int(ns[s]) * int(ks[s]), "uniform", seed=seed * 2_000_003 + s))
    return mats, [int(k) for k in ks], xs


# The benchmark configurations (square lower-triangular, see the header).
def config(name: str, scale: float = 1.0):
    """(matrix, x_true, nrhs) for a named configuration.

    c0      banded n=100,000, 8 off-diagonals in a 256 window, x = 1, seed 0
    c1      2D 5-point lower triangle on 2048x2048, x ~ U(-1,1), seed 1
    c2      Zipf(1.5) DAG n=2,000,000, <=256 off-diagonals, x ~ N(0,1), seed 2
    c2k16   c2 with 16 right-hand sides
    `scale` shrinks n (for tests); scale=1 is the full configuration.
    """
    if name == "c0":
        n = max(16, int(100_000 * scale))
        m = banded(n, 256, 8, 8, seed=0)
        return m, vector(n, "ones"), 1
    if name == "c1":
        g = max(4, int(2048 * scale ** 0.5))
        m = grid2d(g, g, seed=1)
        return m, vector(m.n, "uniform", seed=101), 1
    if name in ("c2", "c2k16"):
        n = max(16, int(2_000_000 * scale))
        k = 16 if name == "c2k16" else 1
        m = zipf(n, 1.5, 256, seed=2)
        return m, vector(n * k, "normal", seed=102), k
    raise KeyError(name)
