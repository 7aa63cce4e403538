"""The CPU oracle, pinned against the reference's known-answer test, against
an independent pure-Python restatement, and against golden vectors produced
by the reference's own kernels (tests/golden/*.npz, see make_golden.py)."""
import numpy as np
import pytest

from conftest import golden_cases, load_golden
from oracle import oracle as O
from sptrsv_b200 import gen


def _matrices():
    return {
        "banded": gen.banded(1500, 64, 2, 12, seed=11),
        "grid": gen.grid2d(40, 30, seed=12),
        "grid3d": gen.grid3d(9, 8, 7, seed=13),
        "zipf": gen.zipf(2500, 1.5, 256, seed=14),
        "block": gen.blockdiag(640, 32, seed=15),
    }


def _py_analysis(rowptr, colidx):
    """Independent pure-Python restatement (small cases only):
    analysis/analysis_csr.cu:104-185 (levels), :12-32 (bucket), :53-57 (key),
    :352 (stable order), :66-102 + :244-270 (warp map)."""
    n = len(rowptr) - 1
    lev = [0] * n
    for i in range(n):
        lev[i] = 1 + max([lev[c] for c in colidx[rowptr[i]:rowptr[i + 1] - 1]], default=0)
    nlevs = max(lev, default=0)

    def bucket(k):
        return 6 if k == 0 else 0 if k == 1 else 1 if k <= 2 else 2 if k <= 4 else 3 if k <= 8 else 4 if k <= 16 else 5

    key = [7 * (lev[i] - 1) + bucket(rowptr[i + 1] - rowptr[i] - 1) for i in range(n)]
    iorder = sorted(range(n), key=lambda i: (key[i], i))
    cnt = [0] * (7 * nlevs)
    for k in key:
        cnt[k] += 1
    ibase, ivect, rows = [], [], 0
    for k in range(7 * nlevs):
        size = 0 if k % 7 == 6 else 2 ** (k % 7)
        sz = size or 1
        nw = -(-cnt[k] * sz // 32)
        for x in range(nw):
            ibase.append(rows + x * (32 // sz))
            ivect.append(size)
        rows += cnt[k]
    ibase.append(n)
    return lev, nlevs, iorder, cnt, ibase, ivect


def test_bucket_table_matches_reference():
    expect = {0: 6, 1: 0, 2: 1, 3: 2, 4: 2, 5: 3, 8: 3, 9: 4, 16: 4, 17: 5, 100: 5}
    for k, b in expect.items():
        assert O.lib().oracle_bucket(k) == b


@pytest.mark.parametrize("name", list(_matrices()))
def test_known_answer_unit_values(name):
    # the reference's own test: every value 1.0, b = row sums, x == 1 exactly
    # (main.cu:228,236; test.cu:10-15; header/matrix_properties.h:14)
    m = _matrices()[name].unit_values()
    b = np.diff(m.rowptr).astype(np.float64)
    x = O.solve(m.rowptr, m.colidx, m.val, b)
    assert np.all(x == 1.0)


@pytest.mark.parametrize("name", list(_matrices()))
def test_fp64_oracle_against_long_double(name):
    m = _matrices()[name]
    xt = gen.vector(m.n, "uniform", seed=3)
    b = m.matvec(xt)
    x = O.solve(m.rowptr, m.colidx, m.val, b)
    xl = O.solve(m.rowptr, m.colidx, m.val, b, long_double=True)
    assert O.rel_err(x, xl) <= 1e-13
    assert O.rel_err(x, xt) <= 1e-12


@pytest.mark.parametrize("name", list(_matrices()))
def test_fp32_restatement(name):
    """The float restatement of the reference's FP32 build: exact on the
    reference's known-answer test, within FP32 accuracy of the FP64 oracle,
    and really computed in float (not the FP64 result rounded)."""
    m = _matrices()[name]
    u = m.unit_values()
    bu = np.diff(u.rowptr).astype(np.float64)
    assert np.all(O.solve(u.rowptr, u.colidx, u.val, bu, f32=True) == 1.0)
    xt = gen.vector(m.n, "uniform", seed=3)
    b = m.matvec(xt)
    x64 = O.solve(m.rowptr, m.colidx, m.val, b)
    x32 = O.solve(m.rowptr, m.colidx, m.val, b, f32=True)
    assert O.rel_err(x32, x64) <= 1e-4
    assert np.array_equal(x32, x32.astype(np.float32).astype(np.float64))
    assert not np.array_equal(x32, x64.astype(np.float32).astype(np.float64)) or m.n < 64


def test_multi_rhs_oracle_matches_single():
    m = _matrices()["zipf"]
    k = 5
    xt = gen.vector(m.n * k, "normal", seed=4)
    b = m.matvec(xt, k)
    x = O.solve(m.rowptr, m.colidx, m.val, b, nrhs=k)
    for j in range(k):
        xj = O.solve(m.rowptr, m.colidx, m.val, np.ascontiguousarray(b[j::k]))
        assert np.array_equal(x[j::k], xj)


def test_level_scheduled_omp_matches_serial():
    m = _matrices()["zipf"]
    a = O.analysis(m.rowptr, m.colidx)
    lev_ptr = np.concatenate([[0], np.cumsum(np.bincount(a["levels"] - 1, minlength=a["nlevs"]))])
    b = m.matvec(gen.vector(m.n, "uniform", seed=9))
    x = O.solve(m.rowptr, m.colidx, m.val, b)
    xo = O.solve_levels_omp(m.rowptr, m.colidx, m.val, b, a["iorder"], lev_ptr, a["nlevs"])
    assert np.array_equal(x, xo)


@pytest.mark.parametrize("seed", range(6))
def test_c_oracle_matches_python_restatement(seed):
    rng = np.random.default_rng(seed)
    n = int(rng.integers(1, 120))
    rows, cols = [0], []
    for i in range(n):
        k = int(rng.integers(0, min(i, 40) + 1)) if i else 0
        c = sorted(rng.choice(i, size=k, replace=False).tolist()) if k else []
        cols += c + [i]
        rows.append(len(cols))
    rp, ci = np.array(rows, np.int32), np.array(cols, np.int32)
    a = O.analysis(rp, ci)
    lev, nlevs, iorder, cnt, ibase, ivect = _py_analysis(rows, cols)
    assert a["nlevs"] == nlevs
    assert a["levels"].tolist() == lev
    assert a["iorder"].tolist() == iorder
    assert a["buckets"].tolist() == cnt
    assert a["ibase_row"].tolist() == ibase
    assert a["ivect_size_warp"].tolist() == ivect
    assert a["n_warps"] == len(ivect)


def test_analysis_edge_cases():
    # n = 1 (diagonal only): one level, one diagonal-only warp
    a = O.analysis(np.array([0, 1]), np.array([0]))
    assert a["nlevs"] == 1 and a["iorder"].tolist() == [0]
    assert a["ivect_size_warp"].tolist() == [0] and a["ibase_row"].tolist() == [0, 1]
    # a pure chain: n levels
    n = 50
    rp = np.concatenate([[0, 1], 1 + 2 * np.arange(1, n)]).astype(np.int32)
    ci = np.concatenate([[0]] + [[i - 1, i] for i in range(1, n)]).astype(np.int32)
    a = O.analysis(rp, ci)
    assert a["nlevs"] == n and a["iorder"].tolist() == list(range(n))


GOLDEN = golden_cases()


@pytest.mark.skipif(not GOLDEN, reason="no golden fixtures")
@pytest.mark.parametrize("path", GOLDEN, ids=[p.stem for p in GOLDEN])
def test_oracle_matches_reference_golden(path):
    g = load_golden(path)
    a = O.analysis(g["rowptr"], g["colidx"])
    assert a["nlevs"] == int(g["ref_nlevs"])
    assert np.array_equal(a["levels"], g["ref_levels"])
    assert np.array_equal(a["iorder"], g["ref_iorder"])
    assert a["n_warps"] == int(g["ref_n_warps"])
    assert np.array_equal(a["ibase_row"], g["ref_ibase_row"])
    assert np.array_equal(a["ivect_size_warp"], g["ref_ivect_size_warp"])
    x = O.solve(g["rowptr"], g["colidx"], g["val"], g["b"])
    for v in ("simple", "order", "multirow"):
        k = f"ref_x_{v}"
        if k in g:
            assert O.rel_err(g[k], x) <= 1e-12, v
    if "ref_x_unit_multirow" in g:
        for v in ("simple", "order", "multirow"):
            assert np.all(g[f"ref_x_unit_{v}"] == 1.0), v


@pytest.mark.parametrize("name,scale", [("c0", 0.05), ("c1", 0.01), ("c2", 0.002), ("c2k16", 0.002)])
def test_oracle_workloads_match_library_generators(name, scale):
    """The CPU baseline builds its inputs through the oracle library; they must
    be the very matrices and vectors the GPU arm solves."""
    from oracle import workloads as W

    m1, x1, k1 = gen.config(name, scale)
    m2, x2, k2 = W.config(name, scale)
    assert k1 == k2
    for a, b in ((m1.rowptr, m2.rowptr), (m1.colidx, m2.colidx), (m1.val, m2.val), (x1, x2)):
        assert np.array_equal(a, b)
    assert np.array_equal(m1.matvec(x1, k1), m2.matvec(x2, k2))


def test_oracle_batch_workload_matches_library_generator():
    from oracle import workloads as W

    a = gen.batch_config(6, seed=3, n_hi=3000)
    b = W.batch_config(6, seed=3, n_hi=3000)
    assert a[1] == b[1]
    for m1, m2, x1, x2 in zip(a[0], b[0], a[2], b[2]):
        assert np.array_equal(m1.rowptr, m2.rowptr) and np.array_equal(m1.colidx, m2.colidx)
        assert np.array_equal(m1.val, m2.val) and np.array_equal(x1, x2)
