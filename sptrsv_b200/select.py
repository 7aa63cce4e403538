"""Schedule selection: analysis features, the exhaustive autotuner and the
learned selector (MLP 12 -> 64 -> 64 -> 24), over the C ABI.

The MLP's forward, backward and Adam kernels run on the GPU inside
libsptrsv_b200.so; this module only moves host arrays in and out.
"""
from __future__ import annotations

import ctypes
from ctypes import byref, c_int, c_void_p

import numpy as np

from . import _lib as C
from ._lib import AnalysisInfo, Schedule, SpMat

N_CLASSES = 24
# version of the class table in csrc/tune.cu; weights trained on another
# table are refused (their outputs would name other schedules)
CLASS_TABLE = 2
N_FEATURES = 12
N_PARAMS = 6552
VARIANT_NAMES = ["simple", "order", "multirow", "cluster", "strip", "wave", "band"]
FEATURE_NAMES = ["log2_n", "log2_nnz", "nnz_per_row", "log2_nlevs", "log2_mean_level_width",
                 "log2_max_level_width", "q25_offdiag", "q50_offdiag", "q90_offdiag", "q99_offdiag",
                 "log2_1p_max_offdiag", "frac_diag_only"]


def features(gpu_L: SpMat, info: AnalysisInfo) -> np.ndarray:
    out = np.zeros(N_FEATURES, dtype=np.float32)
    C.check(C.lib().sptrsv_features(byref(gpu_L), byref(info), out.ctypes.data))
    return out


def schedule_from_class(cls: int) -> Schedule:
    s = Schedule()
    C.check(C.lib().sptrsv_schedule_from_class(int(cls), byref(s)))
    return s


def class_name(cls: int) -> str:
    s = schedule_from_class(cls)
    v = VARIANT_NAMES[s.variant]
    part = f"-P{s.partitions}" if s.partitions >= 2 else ""
    if s.variant in (0, 1):
        return f"{v}/rpw{s.rows_per_warp}{part}"
    if s.variant == 4:
        return f"{v}/R{s.rows_per_warp}-bw{s.block_warps}{part}"
    if s.variant == 5:
        return f"{v}/G{s.block_warps}{part}"
    if s.variant == 6:
        return f"{v}{part}"
    if s.variant == 2:
        return f"{v}/bw{s.block_warps}-bo{s.backoff_ns}-wps{s.warps_per_sm}{part}"
    return f"{v}/H{s.band_levels}-B{s.cluster_rows}-rpw{s.rows_per_warp}-bw{s.block_warps}{part}"


def autotune(plan, b, x, nrhs: int = 1, precision: int = 32, reps: int = 3):
    """(best class, times_ms[24]) — times every class, leaves the best set on the plan."""
    times = np.full(N_CLASSES, np.nan, dtype=np.float32)
    best = c_int(-1)
    C.check(C.lib().sptrsv_autotune(plan.handle, b.data_ptr(), x.data_ptr(), nrhs, precision, reps,
                                    times.ctypes.data, byref(best)))
    return best.value, times


class Mlp:
    """The schedule-selector MLP (parameters live on the GPU)."""

    def __init__(self, seed: int = 0):
        h = c_void_p()
        C.check(C.lib().sptrsv_mlp_create(seed, byref(h)))
        self._h = h

    @property
    def handle(self):
        return self._h

    def params(self) -> np.ndarray:
        p = np.empty(N_PARAMS, dtype=np.float32)
        C.check(C.lib().sptrsv_mlp_get_params(self._h, p.ctypes.data))
        return p

    def set_params(self, p: np.ndarray):
        p = np.ascontiguousarray(p, dtype=np.float32)
        assert p.size == N_PARAMS
        C.check(C.lib().sptrsv_mlp_set_params(self._h, p.ctypes.data))

    def set_normalization(self, mean: np.ndarray, std: np.ndarray):
        m = np.ascontiguousarray(mean, dtype=np.float32)
        s = np.ascontiguousarray(std, dtype=np.float32)
        C.check(C.lib().sptrsv_mlp_set_normalization(self._h, m.ctypes.data, s.ctypes.data))

    def normalization(self):
        m = np.empty(N_FEATURES, np.float32)
        s = np.empty(N_FEATURES, np.float32)
        C.check(C.lib().sptrsv_mlp_get_normalization(self._h, m.ctypes.data, s.ctypes.data))
        return m, s

    def forward(self, X: np.ndarray) -> np.ndarray:
        X = np.ascontiguousarray(X, dtype=np.float32).reshape(-1, N_FEATURES)
        Y = np.empty((X.shape[0], N_CLASSES), dtype=np.float32)
        C.check(C.lib().sptrsv_mlp_forward_host(self._h, X.ctypes.data, X.shape[0], Y.ctypes.data))
        return Y

    def gradient(self, X, T, M):
        X = np.ascontiguousarray(X, dtype=np.float32).reshape(-1, N_FEATURES)
        T = np.ascontiguousarray(T, dtype=np.float32).reshape(-1, N_CLASSES)
        M = np.ascontiguousarray(M, dtype=np.float32).reshape(-1, N_CLASSES)
        g = np.empty(N_PARAMS, dtype=np.float32)
        loss = ctypes.c_float(0)
        C.check(C.lib().sptrsv_mlp_gradient_host(self._h, X.ctypes.data, T.ctypes.data, M.ctypes.data, X.shape[0],
                                                 g.ctypes.data, byref(loss)))
        return float(loss.value), g

    def train(self, X, T, M, epochs: int = 200, batch: int = 64, lr: float = 1e-3, seed: int = 0) -> np.ndarray:
        X = np.ascontiguousarray(X, dtype=np.float32).reshape(-1, N_FEATURES)
        T = np.ascontiguousarray(T, dtype=np.float32).reshape(-1, N_CLASSES)
        M = np.ascontiguousarray(M, dtype=np.float32).reshape(-1, N_CLASSES)
        curve = np.zeros(max(epochs, 1), dtype=np.float32)
        C.check(C.lib().sptrsv_mlp_train_host(self._h, X.ctypes.data, T.ctypes.data, M.ctypes.data, X.shape[0],
                                              epochs, batch, ctypes.c_float(lr), seed, curve.ctypes.data))
        return curve[:epochs]

    def predict_class(self, f: np.ndarray) -> int:
        f = np.ascontiguousarray(f, dtype=np.float32)
        c = c_int(-1)
        C.check(C.lib().sptrsv_mlp_predict_class(self._h, f.ctypes.data, byref(c)))
        return c.value

    def select(self, plan, gpu_L: SpMat, info: AnalysisInfo) -> int:
        c = c_int(-1)
        C.check(C.lib().sptrsv_plan_select_schedule(plan.handle, self._h, byref(gpu_L), byref(info), byref(c)))
        return c.value

    def save(self, path):
        m, s = self.normalization()
        np.savez(path, params=self.params(), mean=m, std=s, table=CLASS_TABLE)

    @classmethod
    def load(cls, path) -> "Mlp":
        z = np.load(path)
        table = int(z["table"]) if "table" in z.files else 1
        if table != CLASS_TABLE:
            raise ValueError(f"{path}: weights for class table {table}, the library has table {CLASS_TABLE}")
        net = cls(0)
        net.set_params(z["params"])
        net.set_normalization(z["mean"], z["std"])
        return net

    def close(self):
        if self._h:
            C.lib().sptrsv_mlp_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def targets_from_times(times: np.ndarray):
    """(T, M): T = log2(time / best) per class, M = 1 where the class ran."""
    times = np.asarray(times, dtype=np.float64).reshape(-1, N_CLASSES)
    ok = np.isfinite(times) & (times > 0)
    best = np.where(ok, times, np.inf).min(axis=1, keepdims=True)
    T = np.where(ok, np.log2(np.where(ok, times, 1.0) / best), 0.0)
    return T.astype(np.float32), ok.astype(np.float32)
