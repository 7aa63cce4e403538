"""The allocation-free solve (sptrsv_solve_ir_noalloc) against the plan-based
FP32 + FP64-refinement solve (sptrsv_solve_ir), through the C ABI.

The allocation-free entry point exists for callers that cannot allocate
device memory at solve time (a device heap owned by a pool or an arena, or
a rule against cudaMalloc after start-up); its scratch is a fixed device
array inside the library.  This file is collected last on purpose, so a run
that stops at the first failure has already run every other test; it also
passes on its own in a fresh process.
"""
import ctypes

import numpy as np
import pytest

from oracle import oracle as O
from sptrsv_b200 import gen

pytestmark = pytest.mark.gpu

TOL = 1e-12  # relative forward error (inf-norm), as in the other solve tests


def _noalloc(L, db, dx, iters=2):
    from sptrsv_b200 import _lib

    return _lib.lib().sptrsv_solve_ir_noalloc(ctypes.byref(L), db.data_ptr(), dx.data_ptr(), iters, None)


@pytest.mark.parametrize("make", [lambda: gen.banded(60000, 256, 8, 8, seed=0), lambda: gen.grid2d(300, 250, seed=1),
                                  lambda: gen.zipf(40000, 1.5, 256, seed=2)], ids=["banded", "grid", "zipf"])
def test_noalloc_matches_plan_solve_twice(torch_cuda, make):
    import sptrsv_b200 as S

    torch = torch_cuda
    m = make()
    L = S.allocate_memory(m.rowptr, m.colidx, m.val, m.n)
    info = S.AnalysisInfo()
    info.mode = S.MULTIROW
    assert S.run_analysis(info, L) == 0
    plan = S.Plan(L, info)
    for call in range(2):  # two calls in a row: the shared scratch must not leak state
        xt = gen.vector(m.n, "uniform", seed=10 + call)
        b = m.matvec(xt)
        db = torch.from_numpy(b).cuda()
        ref = torch.empty_like(db)
        plan.solve_ir(db, ref)
        S.sync_status()
        dx = torch.full_like(db, float("nan"))
        assert _noalloc(L, db, dx) == 0
        got = dx.cpu().numpy()
        assert O.rel_err(got, ref.cpu().numpy()) <= TOL, call
        assert O.rel_err(got, O.solve(m.rowptr, m.colidx, m.val, b)) <= TOL, call
    plan.close()
    S.free_device_analysis(L, info)


def test_noalloc_rejects_sizes_beyond_its_scratch(torch_cuda):
    import sptrsv_b200 as S
    from sptrsv_b200 import _lib

    torch = torch_cuda
    n = (1 << 20) + 1
    m = gen.banded(n, 4, 1, 1, seed=3)
    L = S.allocate_memory(m.rowptr, m.colidx, m.val, m.n)
    db = torch.ones(n, dtype=torch.float64, device="cuda")
    dx = torch.empty_like(db)
    assert _noalloc(L, db, dx) == _lib.SPTRSV_ERR_UNSUPPORTED
    assert "scratch limit" in _lib.last_error()[1]
    S.free_device_analysis(L, None)


def _device_csr(torch, rowptr, colidx, val, nnz=None):
    """An sp_mat_t built directly from device tensors, bypassing the host
    check of allocate_memory (the tensors are returned to keep them alive)."""
    from sptrsv_b200 import _lib

    ia = torch.from_numpy(np.ascontiguousarray(rowptr, np.int32)).cuda()
    ja = torch.from_numpy(np.ascontiguousarray(colidx, np.int32)).cuda()
    a = torch.from_numpy(np.ascontiguousarray(val, np.float64)).cuda()
    n = rowptr.shape[0] - 1
    L = _lib.SpMat(n, n, int(rowptr[-1]) if nnz is None else nnz, ia.data_ptr(), ja.data_ptr(), a.data_ptr())
    return L, (ia, ja, a)


def _corrupt(m, kind):
    """A copy of m with one malformed row.  Every planted index stays inside
    the arrays' allocations, so the check is what turns it into an error."""
    rp, ci, va = m.rowptr.copy(), m.colidx.copy(), m.val.copy()
    nnz = None
    if kind == "above_diagonal":  # row 100: an off-diagonal column right of the diagonal
        ci[rp[100]] = 103
    elif kind == "diagonal_not_last":  # row 200: diagonal swapped with the entry before it
        e = rp[201]
        ci[e - 2], ci[e - 1] = ci[e - 1], ci[e - 2]
        va[e - 2], va[e - 1] = va[e - 1], va[e - 2]
    elif kind == "negative_column":
        ci[rp[300]] = -1
    elif kind == "range_beyond_nnz":  # the last rows' entries lie past the nnz the caller states
        nnz = int(rp[-1]) - 10
    return rp, ci, va, nnz


@pytest.mark.parametrize("kind", ["above_diagonal", "diagonal_not_last", "negative_column", "range_beyond_nnz"])
def test_noalloc_rejects_malformed_csr(torch_cuda, kind):
    """The entry point is meant for callers that never went through
    allocate_memory's host check, so its kernels check every row range and
    column before using it; a malformed CSR ends in SPTRSV_ERR_INVALID_CSR and
    the next call on a good matrix still solves correctly."""
    from sptrsv_b200 import _lib

    torch = torch_cuda
    m = gen.banded(5000, 64, 4, 8, seed=21)
    b = m.matvec(gen.vector(m.n, "uniform", seed=22))
    db = torch.from_numpy(b).cuda()
    dx = torch.empty_like(db)
    rp, ci, va, nnz = _corrupt(m, kind)
    L, keep = _device_csr(torch, rp, ci, va, nnz)
    assert _noalloc(L, db, dx) == _lib.SPTRSV_ERR_INVALID_CSR
    torch.cuda.synchronize()
    good, keep2 = _device_csr(torch, m.rowptr, m.colidx, m.val)
    assert _noalloc(good, db, dx) == 0
    assert O.rel_err(dx.cpu().numpy(), O.solve(m.rowptr, m.colidx, m.val, b)) <= TOL
    del keep, keep2
