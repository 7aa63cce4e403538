"""GPU analysis pass: bit-exact against the CPU oracle and the reference's
own arrays (golden fixtures), edge cases, malformed input."""
import ctypes

import numpy as np
import pytest

from conftest import golden_cases, load_golden
from oracle import oracle as O
from sptrsv_b200 import gen

pytestmark = pytest.mark.gpu


def _analyse(S, m, mode):
    L = S.allocate_memory(m.rowptr, m.colidx, m.val, m.n)
    info = S.AnalysisInfo()
    info.mode = mode
    assert S.run_analysis(info, L) == 0
    got = S.analysis_arrays(info, m.n)
    S.free_device_analysis(L, info)
    return got


def _compare(got, ref, warp_map=True):
    assert got["nlevs"] == ref["nlevs"]
    assert np.array_equal(got["levels"], ref["levels"])
    assert np.array_equal(got["iorder"], ref["iorder"])
    if "buckets" in ref:
        assert np.array_equal(got["buckets"], ref["buckets"])
    if warp_map:
        assert got["n_warps"] == ref["n_warps"]
        assert np.array_equal(got["ibase_row"], ref["ibase_row"])
        assert np.array_equal(got["ivect_size_warp"], ref["ivect_size_warp"])


MATS = {
    "banded": lambda: gen.banded(20000, 256, 8, 8, seed=0),
    "banded_var": lambda: gen.banded(7777, 64, 0, 20, seed=5),
    "grid2d": lambda: gen.grid2d(200, 150, seed=1),
    "grid3d": lambda: gen.grid3d(30, 20, 25, seed=3),
    "zipf": lambda: gen.zipf(50000, 1.5, 256, seed=2),
    "block": lambda: gen.blockdiag(4000, 32, seed=4),
    "single": lambda: gen.from_arrays([0, 1], [0], [3.0]),
    "diag_only": lambda: gen.from_arrays(np.arange(1001), np.arange(1000), np.ones(1000)),
}


@pytest.mark.parametrize("name", list(MATS))
def test_analysis_bit_exact_vs_oracle(torch_cuda, name):
    import sptrsv_b200 as S

    m = MATS[name]()
    ref = O.analysis(m.rowptr, m.colidx)
    got = _analyse(S, m, S.MULTIROW)
    _compare(got, ref)
    assert np.array_equal(got["warp_lev"], ref["warp_lev"])
    assert np.array_equal(got["lev_size"], np.bincount(ref["levels"] - 1, minlength=ref["nlevs"]))
    assert np.array_equal(got["inv_iorder"][got["iorder"]], np.arange(m.n))
    got1 = _analyse(S, m, S.ORDER)  # ORDER fills no warp map in info, like the reference
    _compare(got1, ref, warp_map=False)
    assert got1["n_warps"] == 0 and "ibase_row" not in got1


def test_analysis_chain_deep(torch_cuda):
    import sptrsv_b200 as S

    n = 20000
    rp = np.concatenate([[0, 1], 1 + 2 * np.arange(1, n)])
    ci = np.concatenate([[0]] + [[i - 1, i] for i in range(1, n)])
    m = gen.from_arrays(rp, ci, np.ones(ci.shape[0]))
    got = _analyse(S, m, S.MULTIROW)
    assert got["nlevs"] == n and np.array_equal(got["iorder"], np.arange(n))


@pytest.mark.parametrize("cfg", ["c1", "c2"])
def test_analysis_full_size_configs(torch_cuda, cfg):
    import sptrsv_b200 as S

    m = gen.config(cfg)[0]
    ref = O.analysis(m.rowptr, m.colidx)
    got = _analyse(S, m, S.ALL)
    _compare(got, ref)


GOLDEN = golden_cases()


@pytest.mark.skipif(not GOLDEN, reason="no golden fixtures")
@pytest.mark.parametrize("path", GOLDEN, ids=[p.stem for p in GOLDEN])
def test_analysis_matches_reference_golden(torch_cuda, path):
    import sptrsv_b200 as S

    g = load_golden(path)
    m = gen.from_arrays(g["rowptr"], g["colidx"], g["val"])
    got = _analyse(S, m, S.MULTIROW)
    ref = {"nlevs": int(g["ref_nlevs"]), "levels": g["ref_levels"], "iorder": g["ref_iorder"],
           "n_warps": int(g["ref_n_warps"]), "ibase_row": g["ref_ibase_row"],
           "ivect_size_warp": g["ref_ivect_size_warp"]}
    _compare(got, ref)
    assert np.array_equal(_analyse(S, m, S.ORDER)["iorder"], g["ref_iorder_ordermode"])


def test_malformed_device_csr_is_an_error_not_a_hang(torch_cuda):
    import sptrsv_b200 as S

    torch = torch_cuda
    # row 2 has a column >= its row index; device-side validation must reject it
    rp = torch.tensor([0, 1, 3, 5], dtype=torch.int32, device="cuda")
    ci = torch.tensor([0, 0, 1, 2, 2], dtype=torch.int32, device="cuda")
    va = torch.ones(5, dtype=torch.float64, device="cuda")
    L = S.SpMat(3, 3, 5, rp.data_ptr(), ci.data_ptr(), va.data_ptr())
    info = S.AnalysisInfo()
    info.mode = S.MULTIROW
    with pytest.raises(S.SptrsvError) as e:
        S.run_analysis(info, L)
    assert e.value.code == -3 and "row 2" in str(e.value)
    # missing diagonal in row 1
    ci2 = torch.tensor([0, 0, 0, 1, 2], dtype=torch.int32, device="cuda")
    L2 = S.SpMat(3, 3, 5, rp.data_ptr(), ci2.data_ptr(), va.data_ptr())
    with pytest.raises(S.SptrsvError):
        S.run_analysis(info, L2)


def test_run_analysis_simple_returns_minus_one(torch_cuda):
    import sptrsv_b200 as S

    m = gen.banded(100, 8, 1, 3, seed=1)
    L = S.allocate_memory(m.rowptr, m.colidx, m.val, m.n)
    info = S.AnalysisInfo()
    info.mode = S.SIMPLE
    assert S.run_analysis(info, L) == -1
    S.free_device_analysis(L, None)


def test_bounded_wait_times_out_and_context_survives(torch_cuda):
    import sptrsv_b200 as S
    from sptrsv_b200 import _lib

    r = _lib.lib().sptrsv_selftest_bounded_wait(ctypes.c_ulonglong(50_000_000))  # 50 ms
    assert r == _lib.SPTRSV_ERR_TIMEOUT
    m = gen.banded(3000, 32, 1, 6, seed=9)
    got = _analyse(S, m, S.MULTIROW)
    _compare(got, O.analysis(m.rowptr, m.colidx))


@pytest.mark.parametrize("mode_name", ["ORDER", "MULTIROW"])
def test_multirow_analysis_base_gpu_entry_point(torch_cuda, mode_name):
    """header/analysis.h:20 called by its own name: bit-exact with the oracle
    and with run_analysis, and analysing into the same struct again releases
    the arrays the struct held (no device memory leaks across re-analyses)."""
    import sptrsv_b200 as S

    torch = torch_cuda
    mode = getattr(S, mode_name)
    m = gen.banded(200_000, 256, 8, 8, seed=31)
    ref = O.analysis(m.rowptr, m.colidx)
    L = S.allocate_memory(m.rowptr, m.colidx, m.val, m.n)
    info = S.AnalysisInfo()
    S.multirow_analysis_base_GPU(info, L, mode)
    assert info.mode == mode
    got = S.analysis_arrays(info, m.n)
    _compare(got, ref, warp_map=mode == S.MULTIROW)
    assert np.array_equal(got["iorder"], _analyse(S, m, mode)["iorder"])
    # the same struct analysed again, several times: device memory stays flat
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for _ in range(6):
        S.multirow_analysis_base_GPU(info, L, mode)
    torch.cuda.synchronize()
    free1 = torch.cuda.mem_get_info()[0]
    assert free0 - free1 < 4 << 20, (free0, free1)
    _compare(S.analysis_arrays(info, m.n), ref, warp_map=mode == S.MULTIROW)
    # a plan built on the re-analysed struct solves correctly
    b = m.matvec(gen.vector(m.n, "uniform", seed=32))
    x = np.zeros(m.n)
    S.run_solver(L, info, b, x, m.n)
    assert O.rel_err(x, O.solve(m.rowptr, m.colidx, m.val, b)) <= 1e-12
    S.free_device_analysis(L, info)
