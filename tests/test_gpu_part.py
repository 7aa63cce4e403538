"""Partitioned solves (schedule.partitions >= 2): the rows cut into blocks
solved independently after a warm-up, through the C ABI, against the CPU
oracle — every variant on the block system, FP64 and FP32 + FP64
refinement, several right-hand sides, value updates, host buffers — plus
the block table's invariants and the refusal of matrices that are not
diagonally dominant."""
import numpy as np
import pytest

from oracle import oracle as O
from sptrsv_b200 import gen

pytestmark = pytest.mark.gpu

TOL = 1e-12  # relative forward error (inf-norm) against the FP64 oracle
BOUND = 2.0 ** -60  # the truncation bound every block must meet

MATS = {
    "banded": lambda: gen.banded(30000, 256, 8, 8, seed=0),
    "banded_narrow": lambda: gen.banded(40000, 16, 4, 16, seed=11),
    "grid2d": lambda: gen.grid2d(160, 140, seed=1),
    "grid3d": lambda: gen.grid3d(25, 20, 22, seed=3),
    "zipf": lambda: gen.zipf(40000, 1.5, 256, seed=2),
}


def _setup(S, m):
    L = S.allocate_memory(m.rowptr, m.colidx, m.val, m.n)
    info = S.AnalysisInfo()
    info.mode = S.ALL
    assert S.run_analysis(info, L) == 0
    return L, info


def _check_table(info, n):
    t = info["table"]
    assert t.shape == (info["blocks"], 4)
    s, a, e, base = t[:, 0], t[:, 1], t[:, 2], t[:, 3]
    assert a[0] == 0 and s[0] == 0 and e[-1] == n
    assert np.all(e[:-1] == a[1:]) and np.all(a < e) and np.all((0 <= s) & (s <= a))
    assert np.array_equal(base, np.concatenate([[0], np.cumsum(e - s)[:-1]]))
    assert info["n_ext"] == int((e - s).sum())
    assert info["warm_rows"] == int((a - s).sum())
    assert 0.0 <= info["bound"] <= BOUND


SCHEDS = {
    "multirow": dict(variant=2),
    "order8": dict(variant=1, rows_per_warp=8),
    "simple": dict(variant=0, rows_per_warp=32),
    "cluster": dict(variant=3, rows_per_warp=16, band_levels=256, cluster_rows=2048, block_warps=16),
}


@pytest.mark.parametrize("name", list(MATS))
@pytest.mark.parametrize("P", [2, 7, 32])
def test_partitioned_variants_fp64_and_ir(torch_cuda, name, P):
    import sptrsv_b200 as S

    torch = torch_cuda
    m = MATS[name]()
    xt = gen.vector(m.n, "uniform", seed=9)
    b = m.matvec(xt)
    ref = O.solve(m.rowptr, m.colidx, m.val, b)
    L, info = _setup(S, m)
    plan = S.Plan(L, info)
    db = torch.from_numpy(b).cuda()
    dx = torch.empty(m.n, dtype=torch.float64, device="cuda")
    scheds = list(SCHEDS.values())
    if name.startswith("grid"):
        scheds += [dict(variant=S._lib.VAR_WAVE, block_warps=8), dict(variant=S._lib.VAR_STRIP, rows_per_warp=1)]
    for sc in scheds:
        plan.set_schedule(ir_max_iters=2, partitions=P, **sc)
        _check_table(plan.partition_info(), m.n)
        plan.solve_f64(db, dx)
        S.sync_status()
        assert O.rel_err(dx.cpu().numpy(), ref) <= TOL, (sc, P)
        dx.fill_(0)
        plan.solve_ir(db, dx)
        S.sync_status()
        assert O.rel_err(dx.cpu().numpy(), ref) <= TOL, ("ir", sc, P)
    plan.close()
    S.free_device_analysis(L, info)


def test_partitioned_warmup_bounds_the_dropped_rows(torch_cuda):
    """Block 0 is exact; every other block starts early, and solving the
    block system alone (its real rows kept) matches the full solve."""
    import sptrsv_b200 as S

    torch = torch_cuda
    m = gen.grid2d(200, 300, seed=5)
    xt = gen.vector(m.n, "uniform", seed=3)
    b = m.matvec(xt)
    ref = O.solve(m.rowptr, m.colidx, m.val, b)
    L, info = _setup(S, m)
    plan = S.Plan(L, info)
    plan.set_schedule(variant=S._lib.VAR_WAVE, block_warps=8, partitions=6)
    pi = plan.partition_info()
    _check_table(pi, m.n)
    t = pi["table"]
    assert np.all(t[1:, 0] < t[1:, 1])  # every later block has a warm-up
    # the warm-up covers many grid lines (same-sign neighbours decay by about
    # a third per line) and starts at a line start
    assert np.all(t[1:, 1] - t[1:, 0] >= 20 * 200)
    assert np.all(t[1:, 0] % 200 == 0) and np.all(t[1:, 1] % 200 == 0)
    db = torch.from_numpy(b).cuda()
    dx = torch.empty(m.n, dtype=torch.float64, device="cuda")
    plan.solve_f64(db, dx)
    S.sync_status()
    assert O.rel_err(dx.cpu().numpy(), ref) <= 1e-14
    plan.close()
    S.free_device_analysis(L, info)


@pytest.mark.parametrize("k", [2, 5, 16])
def test_partitioned_multi_rhs(torch_cuda, k):
    import sptrsv_b200 as S

    torch = torch_cuda
    m = gen.banded(20000, 128, 4, 12, seed=12)
    xt = gen.vector(m.n * k, "normal", seed=13)
    b = m.matvec(xt, k)
    ref = O.solve(m.rowptr, m.colidx, m.val, b, nrhs=k)
    L, info = _setup(S, m)
    plan = S.Plan(L, info)
    plan.set_schedule(variant=S._lib.VAR_MULTIROW, ir_max_iters=2, partitions=8)
    db = torch.from_numpy(b).cuda()
    dx = torch.empty(m.n * k, dtype=torch.float64, device="cuda")
    plan.solve_f64(db, dx, k)
    S.sync_status()
    assert O.rel_err(dx.cpu().numpy(), ref) <= TOL
    plan.solve_ir(db, dx, k)
    S.sync_status()
    assert O.rel_err(dx.cpu().numpy(), ref) <= TOL
    plan.close()
    S.free_device_analysis(L, info)


def test_partitioned_value_update_and_host_buffers(torch_cuda):
    import sptrsv_b200 as S

    torch = torch_cuda
    m = gen.banded(25000, 256, 8, 8, seed=21)
    L, info = _setup(S, m)
    plan = S.Plan(L, info)
    plan.set_schedule(variant=S._lib.VAR_CLUSTER, rows_per_warp=16, band_levels=256, cluster_rows=2048,
                      block_warps=16, partitions=16)
    # new values, same pattern: the warm-ups are recomputed for them
    m2 = gen.HostCsr(m.rowptr, m.colidx, m.val.copy())
    rng = np.random.default_rng(4)
    m2.val[m2.rowptr[1:] - 1] *= rng.uniform(1.0, 3.0, m.n)
    L2 = S.allocate_memory(m2.rowptr, m2.colidx, m2.val, m2.n)
    plan.update_values(L2)
    _check_table(plan.partition_info(), m.n)
    xt = gen.vector(m.n, "uniform", seed=22)
    b = m2.matvec(xt)
    ref = O.solve(m2.rowptr, m2.colidx, m2.val, b)
    hx = np.zeros(m.n)
    for prec in (64, 32):
        plan.solve_host(b, hx, 1, precision=prec)
        assert O.rel_err(hx, ref) <= TOL, prec
    db = torch.from_numpy(b).cuda()
    dx = torch.empty(m.n, dtype=torch.float64, device="cuda")
    plan.solve_f64(db, dx)
    S.sync_status()
    assert O.rel_err(dx.cpu().numpy(), ref) <= TOL
    plan.close()
    S.free_device_analysis(L2, None)
    S.free_device_analysis(L, info)


def test_partitioned_needs_diagonal_dominance(torch_cuda):
    import sptrsv_b200 as S

    m = gen.banded(5000, 64, 4, 8, seed=1).unit_values()  # |L_ii| = 1 < row count
    L, info = _setup(S, m)
    plan = S.Plan(L, info)
    with pytest.raises(S.SptrsvError) as ei:
        plan.set_schedule(variant=S._lib.VAR_MULTIROW, partitions=4)
    assert ei.value.code == -9  # SPTRSV_ERR_UNSUPPORTED
    # the plan keeps its previous schedule and still solves
    b = np.diff(m.rowptr).astype(np.float64)
    x = np.zeros(m.n)
    plan.solve_host(b, x, 1, precision=64)
    assert np.array_equal(x, np.ones(m.n))
    with pytest.raises(S.SptrsvError):
        plan.set_schedule(variant=S._lib.VAR_MULTIROW, partitions=5000)  # P > 4096
    plan.close()
    S.free_device_analysis(L, info)


BAND_MATS = {
    "banded": lambda: gen.banded(30000, 256, 8, 8, seed=0),
    "banded_narrow": lambda: gen.banded(20000, 16, 4, 16, seed=11),
    "banded_var": lambda: gen.banded(9000, 64, 0, 24, seed=5),
    "grid2d_small": lambda: gen.grid2d(100, 70, seed=1),
    "chain": lambda: gen.banded(8000, 1, 1, 1, seed=2),
}


@pytest.mark.parametrize("name", list(BAND_MATS))
@pytest.mark.parametrize("P", [0, 5, 24])
def test_band_schedule(torch_cuda, name, P):
    """One warp per unit (the whole matrix, or each block), level by level:
    FP64 and FP32 + refinement, on device and host buffers."""
    import sptrsv_b200 as S

    torch = torch_cuda
    m = BAND_MATS[name]()
    xt = gen.vector(m.n, "uniform", seed=19)
    b = m.matvec(xt)
    ref = O.solve(m.rowptr, m.colidx, m.val, b)
    L, info = _setup(S, m)
    plan = S.Plan(L, info)
    plan.set_schedule(variant=S._lib.VAR_BAND, ir_max_iters=2, partitions=P)
    if P:
        _check_table(plan.partition_info(), m.n)
    db = torch.from_numpy(b).cuda()
    dx = torch.empty(m.n, dtype=torch.float64, device="cuda")
    for _ in range(2):  # the records' b is rewritten by every solve
        plan.solve_f64(db, dx)
        S.sync_status()
        assert O.rel_err(dx.cpu().numpy(), ref) <= TOL, (name, P)
        dx.fill_(0)
        plan.solve_ir(db, dx)
        S.sync_status()
        assert O.rel_err(dx.cpu().numpy(), ref) <= TOL, ("ir", name, P)
    x32 = torch.empty(m.n, dtype=torch.float32, device="cuda")
    plan.solve_f32(db, x32)
    S.sync_status()
    ref32 = O.solve(m.rowptr, m.colidx, m.val, b, f32=True)
    assert O.rel_err(x32.double().cpu().numpy(), ref) <= 1e-4
    assert O.rel_err(x32.double().cpu().numpy(), ref32) <= 1e-4
    hx = np.zeros(m.n)
    plan.solve_host(b, hx, 1, precision=64)
    assert O.rel_err(hx, ref) <= TOL
    plan.close()
    S.free_device_analysis(L, info)


def test_band_unit_values_exact(torch_cuda):
    # the reference's known-answer input: values 1, b = row counts, x == 1 exactly
    import sptrsv_b200 as S

    m = gen.banded(6000, 64, 2, 6, seed=8).unit_values()
    L, info = _setup(S, m)
    plan = S.Plan(L, info)
    plan.set_schedule(variant=S._lib.VAR_BAND)
    b = np.diff(m.rowptr).astype(np.float64)
    x = np.zeros(m.n)
    plan.solve_host(b, x, 1, precision=64)
    assert np.array_equal(x, np.ones(m.n))
    plan.close()
    S.free_device_analysis(L, info)


def test_band_refuses_wide_levels(torch_cuda):
    import sptrsv_b200 as S

    m = gen.blockdiag(8192, 32, seed=4)  # 256 rows per level
    L, info = _setup(S, m)
    plan = S.Plan(L, info)
    with pytest.raises(S.SptrsvError) as ei:
        plan.set_schedule(variant=S._lib.VAR_BAND)
    assert ei.value.code == -9
    plan.close()
    S.free_device_analysis(L, info)


def test_partitioned_wave_streamed_host_solve(torch_cuda):
    """Pinned host b and x with a partitioned WAVE plan: b is copied in
    segments while the block system's kernel runs (warm-up rows read the
    outer b), and each line group's real rows go straight to the host x."""
    import sptrsv_b200 as S

    torch = torch_cuda
    m = gen.grid2d(600, 500, seed=7)
    xt = gen.vector(m.n, "uniform", seed=8)
    b = m.matvec(xt)
    ref = O.solve(m.rowptr, m.colidx, m.val, b)
    L, info = _setup(S, m)
    plan = S.Plan(L, info)
    hb = torch.from_numpy(b).pin_memory()
    hx = torch.zeros(m.n, dtype=torch.float64).pin_memory()
    for P, G in ((16, 4), (5, 8)):
        plan.set_schedule(variant=S._lib.VAR_WAVE, block_warps=G, partitions=P)
        for _ in range(3):  # epochs advance from call to call
            hx.zero_()
            plan.solve_host(hb, hx, 1, precision=64)
            assert O.rel_err(hx.numpy(), ref) <= TOL, (P, G)
    plan.close()
    S.free_device_analysis(L, info)
