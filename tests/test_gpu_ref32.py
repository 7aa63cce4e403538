"""Parity with the reference's FP32 build (VALUE_TYPE = float, Makefile:7):
the library's FP32 solve against the oracle's float restatement of the
reference substitution on the same matrix, and both against the FP64 oracle.
(The reference's float build itself is not run on the GPU: its first run
aborted inside the reference's solver.)"""
import numpy as np
import pytest

from oracle import oracle as O
from sptrsv_b200 import gen

pytestmark = pytest.mark.gpu

F32_TOL = 1e-4  # relative forward error of an FP32 substitution on these diagonally dominant systems


@pytest.mark.parametrize("make", [lambda: gen.banded(3000, 64, 2, 10, seed=31), lambda: gen.grid2d(50, 40, seed=32),
                                  lambda: gen.zipf(4000, 1.5, 256, seed=33)], ids=["banded", "grid", "zipf"])
def test_fp32_solve_matches_float_restatement(torch_cuda, make):
    import sptrsv_b200 as S

    torch = torch_cuda
    m = make()
    xt = gen.vector(m.n, "uniform", seed=34)
    b = m.matvec(xt)
    ref64 = O.solve(m.rowptr, m.colidx, m.val, b)
    ref32 = O.solve(m.rowptr, m.colidx, m.val, b, f32=True)
    assert O.rel_err(ref32, ref64) <= F32_TOL
    L = S.allocate_memory(m.rowptr, m.colidx, m.val, m.n)
    info = S.AnalysisInfo()
    info.mode = S.MULTIROW
    assert S.run_analysis(info, L) == 0
    plan = S.Plan(L, info)
    db = torch.from_numpy(b).cuda()
    x32 = torch.empty(m.n, dtype=torch.float32, device="cuda")
    for v in (S._lib.VAR_SIMPLE, S._lib.VAR_ORDER, S._lib.VAR_MULTIROW):
        plan.set_schedule(variant=v, rows_per_warp=1)
        plan.solve_f32(db, x32)
        S.sync_status()
        ours = x32.double().cpu().numpy()
        assert O.rel_err(ours, ref64) <= F32_TOL, v
        assert O.rel_err(ours, ref32) <= 2 * F32_TOL, v
    # unit values: both FP32 paths are exact (the reference's own test)
    u = m.unit_values()
    bu = np.diff(u.rowptr).astype(np.float64)
    assert np.all(O.solve(u.rowptr, u.colidx, u.val, bu, f32=True) == 1.0)
    Lu = S.allocate_memory(u.rowptr, u.colidx, u.val, u.n)
    iu = S.AnalysisInfo()
    iu.mode = S.MULTIROW
    S.run_analysis(iu, Lu)
    pu = S.Plan(Lu, iu)
    pu.solve_f32(torch.from_numpy(bu).cuda(), x32)
    S.sync_status()
    assert bool((x32 == 1.0).all())
    pu.close()
    plan.close()
    S.free_device_analysis(Lu, iu)
    S.free_device_analysis(L, info)
