"""The benchmark workloads, generated through the oracle library.

TEST INFRASTRUCTURE ONLY.  The seeded generators of the library
(sptrsv_b200/csrc/gen.cpp) are compiled into oracle/liboracle.so as well, so
that the CPU baseline (bench.py --impl reference) builds exactly the
matrices and right-hand sides the GPU arm solves without importing or
loading the product package.  The configuration parameters below restate
those of sptrsv_b200/gen.py; tests/test_oracle.py checks that both produce
identical arrays.
"""
from __future__ import annotations

import ctypes
from ctypes import POINTER, byref, c_double, c_int, c_longlong, c_uint64, c_void_p
from dataclasses import dataclass

import numpy as np

from . import oracle as O


class _HostCsr(ctypes.Structure):
    _fields_ = [("n", c_int), ("nnz", c_int), ("rowptr", POINTER(c_int)), ("colidx", POINTER(c_int)),
                ("val", POINTER(c_double))]


_bound = False


def _lib():
    global _bound
    L = O.lib()
    if not _bound:
        P = POINTER(_HostCsr)
        L.sptrsv_gen_banded.restype = c_int
        L.sptrsv_gen_banded.argtypes = [c_int, c_int, c_int, c_int, c_uint64, P]
        L.sptrsv_gen_grid2d.restype = c_int
        L.sptrsv_gen_grid2d.argtypes = [c_int, c_int, c_uint64, P]
        L.sptrsv_gen_zipf.restype = c_int
        L.sptrsv_gen_zipf.argtypes = [c_int, c_double, c_int, c_uint64, P]
        L.sptrsv_gen_vector.restype = c_int
        L.sptrsv_gen_vector.argtypes = [c_longlong, c_int, c_uint64, c_void_p]
        L.sptrsv_host_csr_free.restype = None
        L.sptrsv_host_csr_free.argtypes = [P]
        _bound = True
    return L


@dataclass
class Csr:
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
        return O.spmv(self.rowptr, self.colidx, self.val, x, nrhs)


def _take(fn, *args) -> Csr:
    h = _HostCsr()
    rc = fn(*args, byref(h))
    if rc != 0:
        raise RuntimeError(f"generator failed ({rc})")
    try:
        n, nnz = h.n, h.nnz
        rp = np.ctypeslib.as_array(h.rowptr, shape=(n + 1,)).copy()
        ci = np.ctypeslib.as_array(h.colidx, shape=(max(nnz, 1),))[:nnz].copy()
        va = np.ctypeslib.as_array(h.val, shape=(max(nnz, 1),))[:nnz].copy()
    finally:
        _lib().sptrsv_host_csr_free(byref(h))
    return Csr(rp, ci, va)


def banded(n, bandwidth=256, off_min=8, off_max=8, seed=0) -> Csr:
    return _take(_lib().sptrsv_gen_banded, n, bandwidth, off_min, off_max, seed)


def grid2d(nx, ny=None, seed=1) -> Csr:
    return _take(_lib().sptrsv_gen_grid2d, nx, ny if ny is not None else nx, seed)


def zipf(n, s=1.5, max_off=256, seed=2) -> Csr:
    return _take(_lib().sptrsv_gen_zipf, n, s, max_off, seed)


def vector(m, dist="ones", seed=0) -> np.ndarray:
    out = np.empty(m, dtype=np.float64)
    rc = _lib().sptrsv_gen_vector(m, {"ones": 0, "uniform": 1, "normal": 2}[dist], seed, out.ctypes.data)
    if rc != 0:
        raise RuntimeError(f"vector generator failed ({rc})")
    return out


def config(name: str, scale: float = 1.0):
    """(matrix, x_true, nrhs) of a named configuration (c0, c1, c2, c2k16)."""
    if name == "c0":
        n = max(16, int(100_000 * scale))
        return banded(n, 256, 8, 8, seed=0), vector(n, "ones"), 1
    if name == "c1":
        g = max(4, int(2048 * scale ** 0.5))
        m = grid2d(g, g, seed=1)
        return m, vector(m.n, "uniform", seed=101), 1
    if name in ("c2", "c2k16"):
        n = max(16, int(2_000_000 * scale))
        k = 16 if name == "c2k16" else 1
        return zipf(n, 1.5, 256, seed=2), vector(n * k, "normal", seed=102), k
    raise KeyError(name)


def batch_config(nsys=512, seed=3, n_lo=1000, n_hi=200_000, bw_lo=16, bw_hi=4096, off_lo=4, off_hi=16,
                 k_max=32):
    """The batched configuration: (matrices, right-hand-side counts, x_true)."""
    rng = np.random.default_rng(seed)
    ns = np.exp(rng.uniform(np.log(n_lo), np.log(n_hi), nsys)).astype(np.int64)
    bws = np.exp(rng.uniform(np.log(bw_lo), np.log(bw_hi), nsys)).astype(np.int64)
    ks = rng.integers(1, k_max + 1, nsys)
    mats, xs = [], []
    for s in range(nsys):
        mats.append(banded(int(ns[s]), int(bws[s]), off_lo, off_hi, seed=seed * 1_000_003 + s))
        xs.append(vector(int(ns[s]) * int(ks[s]), "uniform", seed=seed * 2_000_003 + s))
    return mats, [int(k) for k in ks], xs
