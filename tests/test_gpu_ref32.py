"""Parity with the reference's FP32 build (VALUE_TYPE = float, Makefile:7):
the library's FP32 solve against the reference's own float solvers run from
oracle/_ref/libsptrsv_ref_f32.so on the same matrix, and both against the
FP64 oracle."""
import numpy as np
import pytest

from oracle import oracle as O
from sptrsv_b200 import gen

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not O.ref_available(f32=True), reason="reference FP32 build not present")]

F32_TOL = 1e-4  # relative forward error of an FP32 substitution on these diagonally dominant systems


@pytest.mark.parametrize("make", [lambda: gen.banded(3000, 64, 2, 10, seed=31), lambda: gen.grid2d(50, 40, seed=32),
                                  lambda: gen.zipf(4000, 1.5, 256, seed=33)], ids=["banded", "grid", "zipf"])
def test_fp32_solve_matches_reference_float_build(torch_cuda, make):
    import sptrsv_b200 as S

    torch = torch_cuda
    m = make()
    xt = gen.vector(m.n, "uniform", seed=34)
    b = m.matvec(xt)
    ref64 = O.solve(m.rowptr, m.colidx, m.val, b)
    L = S.allocate_memory(m.rowptr, m.colidx, m.val, m.n)
    info = S.AnalysisInfo()
    info.mode = S.MULTIROW
    assert S.run_analysis(info, L) == 0
    plan = S.Plan(L, info)
    db = torch.from_numpy(b).cuda()
    x32 = torch.empty(m.n, dtype=torch.float32, device="cuda")
    plan.solve_f32(db, x32)
    S.sync_status()
    ours = x32.double().cpu().numpy()
    assert O.rel_err(ours, ref64) <= F32_TOL
    for variant in (0, 1, 2):
        xr, _ = O.ref_solve(variant, m.rowptr, m.colidx, m.val, b, f32=True)
        assert O.rel_err(xr, ref64) <= F32_TOL, variant
        assert O.rel_err(ours, xr) <= 2 * F32_TOL, variant
    # unit values: both FP32 paths are exact (the reference's own test)
    u = m.unit_values()
    bu = np.diff(u.rowptr).astype(np.float64)
    Lu = S.allocate_memory(u.rowptr, u.colidx, u.val, u.n)
    iu = S.AnalysisInfo()
    iu.mode = S.MULTIROW
    S.run_analysis(iu, Lu)
    pu = S.Plan(Lu, iu)
    pu.solve_f32(torch.from_numpy(bu).cuda(), x32)
    S.sync_status()
    assert bool((x32 == 1.0).all())
    xr, _ = O.ref_solve(2, u.rowptr, u.colidx, u.val, bu, f32=True)
    assert np.all(xr == 1.0)
    pu.close()
    plan.close()
    S.free_device_analysis(Lu, iu)
    S.free_device_analysis(L, info)
