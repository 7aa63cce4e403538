"""Batched solves over the C ABI: many independent systems, each with its own
number of right-hand sides, in one persistent launch (optionally replayed
from a CUDA graph)."""
from __future__ import annotations

from ctypes import byref, c_int, c_longlong, c_void_p

import numpy as np

from . import _lib as C
from ._lib import SpMat
from .interface import _dev, _stream


class Batch:
    def __init__(self, mats: list[SpMat], nrhs):
        arr = (SpMat * len(mats))(*mats)
        k = np.ascontiguousarray(nrhs, dtype=np.int32)
        assert k.shape[0] == len(mats)
        h = c_void_p()
        C.check(C.lib().sptrsv_batch_create(len(mats), arr, k.ctypes.data, byref(h)))
        self._h = h
        self.nsys = len(mats)
        self.nrhs = k
        off = np.zeros(self.nsys + 1, dtype=np.int64)
        n, nl, vl = c_int(0), c_int(0), c_longlong(0)
        C.check(C.lib().sptrsv_batch_info(h, off.ctypes.data, byref(n), byref(nl), byref(vl)))
        self.offsets, self.n, self.nlevs, self.vec_len = off, n.value, nl.value, vl.value

    LEVEL, CHUNK, HYBRID = 0, 1, 2

    def set_schedule(self, mode: int = 2, block_warps: int = 8, warps_per_sm: int = 0, backoff_ns: int = 0,
                     ir_iters: int = 2):
        """mode 0 level-ordered, 1 natural-order chunks, 2 hybrid (near-chain
        systems on one warp each, see set_seq_width)."""
        C.check(C.lib().sptrsv_batch_set_schedule(self._h, mode, block_warps, warps_per_sm, backoff_ns, ir_iters))

    def set_partition(self, block_rows: int):
        """Cut long diagonally dominant systems into blocks of about block_rows
        rows solved independently after a warm-up (0: no cutting)."""
        C.check(C.lib().sptrsv_batch_set_partition(self._h, int(block_rows)))

    def partition_info(self) -> dict:
        cut, inner, warm, bound = c_int(0), c_int(0), c_longlong(0), C.c_double(0)
        C.check(C.lib().sptrsv_batch_partition_info(self._h, byref(cut), byref(inner), byref(warm), byref(bound)))
        return {"systems_cut": cut.value, "inner_systems": inner.value, "warm_rows": warm.value, "bound": bound.value}

    def set_seq_width(self, width: float):
        C.check(C.lib().sptrsv_batch_set_seq_width(self._h, float(width)))

    def seq_systems(self) -> tuple[int, int, int]:
        """(sequential systems, warps they occupy, rows left to the level tasks)."""
        a, w, r = c_int(0), c_int(0), c_int(0)
        C.check(C.lib().sptrsv_batch_seq_systems(self._h, byref(a), byref(w), byref(r)))
        return a.value, w.value, r.value

    def solve(self, b, x, precision: int = 32, stream=None):
        C.check(C.lib().sptrsv_batch_solve(self._h, _dev(b, "float64", self.vec_len), _dev(x, "float64", self.vec_len),
                                           precision, _stream(stream)))

    def solve_graph(self, b, x, precision: int = 32, stream=None):
        C.check(C.lib().sptrsv_batch_solve_graph(self._h, _dev(b, "float64", self.vec_len),
                                                 _dev(x, "float64", self.vec_len), precision, _stream(stream)))

    def close(self):
        if self._h:
            C.lib().sptrsv_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
