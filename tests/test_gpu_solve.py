"""GPU solves through the C ABI: the reference entry points and the plan
path (FP64, FP32 + FP64 refinement, multi-RHS), against the CPU oracle,
the reference's known-answer test and the reference's own solutions."""
import numpy as np
import pytest

from conftest import golden_cases, load_golden
from oracle import oracle as O
from sptrsv_b200 import gen

pytestmark = pytest.mark.gpu

TOL = 1e-12  # relative forward error (inf-norm) against the FP64 oracle


def _setup(S, m, mode=None):
    L = S.allocate_memory(m.rowptr, m.colidx, m.val, m.n)
    info = None
    if mode is not None:
        info = S.AnalysisInfo()
        info.mode = mode
        assert S.run_analysis(info, L) == 0
    return L, info


MATS = {
    "banded": lambda: gen.banded(30000, 256, 8, 8, seed=0),
    "banded_var": lambda: gen.banded(9000, 64, 0, 24, seed=5),
    "grid2d": lambda: gen.grid2d(160, 140, seed=1),
    "grid3d": lambda: gen.grid3d(25, 20, 22, seed=3),
    "zipf": lambda: gen.zipf(40000, 1.5, 256, seed=2),
    "block": lambda: gen.blockdiag(3000, 32, seed=4),
}


@pytest.mark.parametrize("name", list(MATS))
@pytest.mark.parametrize("mode", ["SIMPLE", "ORDER", "MULTIROW", "ALL"])
def test_run_solver_host_buffers(torch_cuda, name, mode):
    import sptrsv_b200 as S

    m = MATS[name]()
    xt = gen.vector(m.n, "uniform", seed=7)
    b = m.matvec(xt)
    ref = O.solve(m.rowptr, m.colidx, m.val, b)
    L, info = _setup(S, m, None if mode == "SIMPLE" else getattr(S, mode))
    x = np.zeros(m.n)
    S.run_solver(L, info, b, x, m.n)
    assert O.rel_err(x, ref) <= TOL
    S.free_device_analysis(L, info)


@pytest.mark.parametrize("name", list(MATS))
def test_known_answer_unit_values_exact(torch_cuda, name):
    # the reference's test input: values 1.0, b = row counts, x == 1 exactly
    import sptrsv_b200 as S

    m = MATS[name]().unit_values()
    b = np.diff(m.rowptr).astype(np.float64)
    L, info = _setup(S, m, S.ALL)
    for inf in (None, info):
        x = np.zeros(m.n)
        S.run_solver(L, inf, b, x, m.n)
        assert np.all(x == 1.0)
    info.mode = S.ORDER
    x = np.zeros(m.n)
    S.run_solver(L, info, b, x, m.n)
    assert np.all(x == 1.0)
    plan = S.Plan(L, info)
    for prec in (64, 32):
        xp = np.zeros(m.n)
        plan.solve_host(b, xp, 1, precision=prec)
        assert np.all(xp == 1.0), prec
    plan.close()
    S.free_device_analysis(L, info)


@pytest.mark.parametrize("name", ["banded_var", "zipf", "grid2d"])
def test_device_entry_points_and_order_tiles(torch_cuda, name):
    import sptrsv_b200 as S

    torch = torch_cuda
    m = MATS[name]()
    xt = gen.vector(m.n, "normal", seed=8)
    b = m.matvec(xt)
    ref = O.solve(m.rowptr, m.colidx, m.val, b)
    L, info = _setup(S, m, S.MULTIROW)
    db = torch.from_numpy(b).cuda()
    dx = torch.empty(m.n, dtype=torch.float64, device="cuda")
    s = torch.cuda.current_stream()
    for fn in (lambda: S.csr_L_solve_simple(L, db, dx, m.n),
               lambda: S.csr_L_solve_order(L, info, db, dx, m.n, s),
               lambda: S.csr_L_solve_multirow(L, info, db, dx, m.n, s)):
        dx.fill_(0)
        fn()
        S.sync_status(s)
        assert O.rel_err(dx.cpu().numpy(), ref) <= TOL
    for tile in (1, 2, 4, 8, 16, 32):
        S.csr_L_solve_order_tile(L, info, db, dx, tile, s)
        S.sync_status(s)
        assert O.rel_err(dx.cpu().numpy(), ref) <= TOL, tile
    S.free_device_analysis(L, info)


@pytest.mark.parametrize("name", list(MATS))
def test_plan_variants_fp64_and_ir(torch_cuda, name):
    import sptrsv_b200 as S

    torch = torch_cuda
    m = MATS[name]()
    xt = gen.vector(m.n, "uniform", seed=9)
    b = m.matvec(xt)
    ref = O.solve(m.rowptr, m.colidx, m.val, b)
    L, info = _setup(S, m, S.MULTIROW)
    plan = S.Plan(L, info)
    db = torch.from_numpy(b).cuda()
    dx = torch.empty(m.n, dtype=torch.float64, device="cuda")
    scheds = [dict(variant=v, rows_per_warp=r) for v in (S._lib.VAR_SIMPLE, S._lib.VAR_ORDER)
              for r in (1, 2, 8, 32)]
    scheds += [dict(variant=S._lib.VAR_MULTIROW, rows_per_warp=1),
               dict(variant=S._lib.VAR_MULTIROW, rows_per_warp=1, block_warps=4, warps_per_sm=16, backoff_ns=200)]
    scheds += [dict(variant=S._lib.VAR_CLUSTER, rows_per_warp=r, band_levels=h, cluster_rows=bsz, block_warps=bw)
               for (r, h, bsz, bw) in ((1, 64, 4096, 8), (2, 16, 1024, 4), (16, 4, 256, 2), (32, 1, 32, 16),
                                       (4, 128, 8192, 16))]
    for sc in scheds:
        plan.set_schedule(ir_max_iters=2, **sc)
        plan.solve_f64(db, dx)
        S.sync_status()
        assert O.rel_err(dx.cpu().numpy(), ref) <= TOL, sc
        plan.solve_ir(db, dx)
        S.sync_status()
        assert O.rel_err(dx.cpu().numpy(), ref) <= TOL, ("ir", sc)
    dr = torch.empty_like(dx)
    plan.residual(db, dx, dr)
    S.sync_status()
    assert float(dr.abs().max()) <= 1e-12 * float(db.abs().max())
    plan.close()
    S.free_device_analysis(L, info)


@pytest.mark.parametrize("k", [1, 2, 3, 8, 16, 32])
def test_plan_multi_rhs(torch_cuda, k):
    import sptrsv_b200 as S

    torch = torch_cuda
    m = gen.zipf(20000, 1.5, 256, seed=2)
    xt = gen.vector(m.n * k, "normal", seed=10)
    b = m.matvec(xt, k)
    ref = O.solve(m.rowptr, m.colidx, m.val, b, nrhs=k)
    L, info = _setup(S, m, S.MULTIROW)
    plan = S.Plan(L, info)
    db = torch.from_numpy(b).cuda()
    dx = torch.empty(m.n * k, dtype=torch.float64, device="cuda")
    plan.solve_f64(db, dx, k)
    S.sync_status()
    assert O.rel_err(dx.cpu().numpy(), ref) <= TOL
    plan.solve_ir(db, dx, k)
    S.sync_status()
    assert O.rel_err(dx.cpu().numpy(), ref) <= TOL
    x = np.zeros(m.n * k)
    plan.solve_host(b, x, k, precision=32)
    assert O.rel_err(x, ref) <= TOL
    plan.close()
    S.free_device_analysis(L, info)


@pytest.mark.parametrize("cfg,k", [("grid", 1), ("zipf", 16)])
def test_calibrated_refinement_meets_tolerance(torch_cuda, cfg, k):
    import sptrsv_b200 as S

    torch = torch_cuda
    m = gen.grid2d(400, 400, seed=1) if cfg == "grid" else gen.zipf(100000, 1.5, 256, seed=2)
    xt = gen.vector(m.n * k, "normal", seed=11)
    b = m.matvec(xt, k)
    L, info = _setup(S, m, S.MULTIROW)
    plan = S.Plan(L, info)
    db = torch.from_numpy(b).cuda()
    dx = torch.empty_like(db)
    iters, est = plan.calibrate_ir(db, dx, k, tol=1e-13, max_iters=4)
    assert 1 <= iters <= 3 and est <= 1e-13
    assert plan.schedule().ir_max_iters == iters
    plan.solve_ir(db, dx, k)
    S.sync_status()
    assert O.rel_err(dx.cpu().numpy(), O.solve(m.rowptr, m.colidx, m.val, b, nrhs=k)) <= TOL
    plan.close()
    S.free_device_analysis(L, info)


def test_value_update_reuses_analysis(torch_cuda):
    import sptrsv_b200 as S

    m = gen.banded(5000, 64, 2, 10, seed=12)
    m2 = gen.from_arrays(m.rowptr, m.colidx, m.val * 1.5)
    b = m2.matvec(gen.vector(m.n, "uniform", seed=3))
    L, info = _setup(S, m, S.MULTIROW)
    plan = S.Plan(L, info)
    L2 = S.allocate_memory(m2.rowptr, m2.colidx, m2.val, m2.n)
    plan.update_values(L2)
    x = np.zeros(m.n)
    plan.solve_host(b, x, 1, precision=64)
    assert O.rel_err(x, O.solve(m2.rowptr, m2.colidx, m2.val, b)) <= TOL
    plan.close()
    S.free_device_analysis(L2, None)
    S.free_device_analysis(L, info)


def test_non_finite_values_complete_without_hanging(torch_cuda):
    import sptrsv_b200 as S

    m = gen.banded(2000, 32, 1, 4, seed=13)
    val = m.val.copy()
    val[m.rowptr[501] - 1] = 0.0  # zero diagonal in row 500 -> inf/nan downstream
    mz = gen.from_arrays(m.rowptr, m.colidx, val)
    b = m.matvec(np.ones(m.n))
    ref = O.solve(mz.rowptr, mz.colidx, mz.val, b)
    L, info = _setup(S, mz, S.MULTIROW)
    for inf in (None, info):
        x = np.zeros(m.n)
        S.run_solver(L, inf, b, x, m.n)
        assert np.array_equal(np.isfinite(x), np.isfinite(ref))
    S.free_device_analysis(L, info)


@pytest.mark.parametrize("cfg", ["c0", "c1", "c2", "c2k16"])
def test_full_size_configs_fp64_and_ir(torch_cuda, cfg):
    import sptrsv_b200 as S

    torch = torch_cuda
    m, xt, k = gen.config(cfg)
    b = m.matvec(xt, k)
    ref = O.solve(m.rowptr, m.colidx, m.val, b, nrhs=k)
    L, info = _setup(S, m, S.MULTIROW)
    plan = S.Plan(L, info)
    db = torch.from_numpy(b).cuda()
    dx = torch.empty(m.n * k, dtype=torch.float64, device="cuda")
    plan.solve_f64(db, dx, k)
    S.sync_status()
    assert O.rel_err(dx.cpu().numpy(), ref) <= TOL
    plan.solve_ir(db, dx, k)
    S.sync_status()
    e = O.rel_err(dx.cpu().numpy(), ref)
    assert e <= TOL, e
    assert O.rel_err(dx.cpu().numpy(), xt) <= TOL
    plan.close()
    S.free_device_analysis(L, info)


GOLDEN = golden_cases()


@pytest.mark.skipif(not GOLDEN, reason="no golden fixtures")
@pytest.mark.parametrize("path", GOLDEN, ids=[p.stem for p in GOLDEN])
def test_solves_match_reference_golden(torch_cuda, path):
    import sptrsv_b200 as S

    g = load_golden(path)
    m = gen.from_arrays(g["rowptr"], g["colidx"], g["val"])
    L, info = _setup(S, m, S.MULTIROW)
    for mode, inf in (("simple", None), ("multirow", info)):
        x = np.zeros(m.n)
        S.run_solver(L, inf, g["b"], x, m.n)
        for v in ("simple", "order", "multirow"):
            assert O.rel_err(x, g[f"ref_x_{v}"]) <= TOL, (mode, v)
    plan = S.Plan(L, info)
    x = np.zeros(m.n)
    plan.solve_host(np.ascontiguousarray(g["b"]), x, 1, precision=32)
    assert O.rel_err(x, g["ref_x_multirow"]) <= TOL
    plan.close()
    S.free_device_analysis(L, info)


STRIP_OK = {
    "grid2d_aligned": lambda: gen.grid2d(160, 140, seed=1),
    "grid2d_ragged": lambda: gen.grid2d(100, 77, seed=2),
    "grid3d": lambda: gen.grid3d(40, 20, 15, seed=3),
    "grid3d_ragged": lambda: gen.grid3d(45, 13, 9, seed=4),
    "grid2d_short_lines": lambda: gen.grid2d(20, 90, seed=5),
    "grid2d_long_lines": lambda: gen.grid2d(4000, 6, seed=6),
    "uneven_lines": lambda: _uneven_lines(300, seed=7),
}


def _uneven_lines(nlines, seed):
    """Lines of random lengths (1..150 rows): every row but a line's first
    depends on the row before it, and most rows on the row at the same offset
    of the line before when that line is long enough (the structure of a 2D
    stencil on a ragged domain)."""
    rng = np.random.default_rng(seed)
    lens = rng.integers(1, 151, size=nlines)
    starts = np.concatenate([[0], np.cumsum(lens)])
    rowptr, cols, vals = [0], [], []
    for li in range(nlines):
        for o in range(int(lens[li])):
            i = int(starts[li]) + o
            row = []
            if li > 0 and o < lens[li - 1] and rng.random() < 0.9:
                row.append(int(starts[li - 1]) + o)
            if o > 0:
                row.append(i - 1)
            off = rng.uniform(-0.5, 0.5, size=len(row))
            cols += row + [i]
            vals += list(off) + [1.0 + float(np.abs(off).sum())]
            rowptr.append(len(cols))
    return gen.HostCsr(np.array(rowptr, dtype=np.int32), np.array(cols, dtype=np.int32),
                       np.array(vals, dtype=np.float64))


@pytest.mark.parametrize("name", list(STRIP_OK))
def test_strip_schedule_fp64_and_ir(torch_cuda, name):
    """The STRIP schedule (prefix scan over 32-row chunks, grid lines per warp
    in wavefront order) against the oracle, for several lines per warp."""
    import sptrsv_b200 as S

    torch = torch_cuda
    m = STRIP_OK[name]()
    xt = gen.vector(m.n, "uniform", seed=9)
    b = m.matvec(xt)
    ref = O.solve(m.rowptr, m.colidx, m.val, b)
    L, info = _setup(S, m, S.MULTIROW)
    plan = S.Plan(L, info)
    db = torch.from_numpy(b).cuda()
    dx = torch.empty(m.n, dtype=torch.float64, device="cuda")
    scheds = [dict(variant=S._lib.VAR_STRIP, rows_per_warp=r, block_warps=bw)
              for r, bw in ((1, 4), (2, 2), (4, 4), (8, 4), (16, 4), (32, 2))]
    # 4000-row lines: a group of more than 4 does not fit shared memory
    gs = (2, 4) if name == "grid2d_long_lines" else (2, 4, 8, 16)
    scheds += [dict(variant=S._lib.VAR_WAVE, block_warps=g) for g in gs]
    for sc in scheds:
        plan.set_schedule(ir_max_iters=2, **sc)
        for rep in range(2):
            plan.solve_f64(db, dx)
            S.sync_status()
            assert O.rel_err(dx.cpu().numpy(), ref) <= TOL, (sc, rep)
        plan.solve_ir(db, dx)
        S.sync_status()
        assert O.rel_err(dx.cpu().numpy(), ref) <= TOL, ("ir", sc)
    # new values, same pattern: the strip copy is rebuilt
    m2 = gen.HostCsr(m.rowptr, m.colidx, m.val * 1.5)
    L2 = S.allocate_memory(m2.rowptr, m2.colidx, m2.val, m2.n)
    plan.update_values(L2)
    plan.solve_f64(db, dx)
    S.sync_status()
    assert O.rel_err(dx.cpu().numpy(), ref / 1.5) <= TOL
    plan.close()
    S.free_device_analysis(L2, None)
    S.free_device_analysis(L, info)


@pytest.mark.parametrize("name", ["banded", "zipf"])
def test_strip_schedule_rejects_other_structures(torch_cuda, name):
    import sptrsv_b200 as S

    m = gen.banded(5000, 64, 4, 8, seed=1) if name == "banded" else gen.zipf(5000, 1.5, 64, seed=1)
    L, info = _setup(S, m, S.MULTIROW)
    plan = S.Plan(L, info)
    for v in (S._lib.VAR_STRIP, S._lib.VAR_WAVE):
        with pytest.raises(S.SptrsvError) as ei:
            plan.set_schedule(variant=v, rows_per_warp=4, block_warps=4)
        assert ei.value.code == S._lib.SPTRSV_ERR_UNSUPPORTED
    plan.close()
    S.free_device_analysis(L, info)


def test_wave_schedule_rejects_groups_beyond_shared_memory(torch_cuda):
    import sptrsv_b200 as S

    torch = torch_cuda
    m = gen.grid2d(10000, 20, seed=1)  # 16 lines of 10,000 rows do not fit shared memory; 2 lines do
    L, info = _setup(S, m, S.MULTIROW)
    plan = S.Plan(L, info)
    with pytest.raises(S.SptrsvError) as ei:
        plan.set_schedule(variant=S._lib.VAR_WAVE, block_warps=16)
    assert ei.value.code == S._lib.SPTRSV_ERR_UNSUPPORTED
    xt = gen.vector(m.n, "uniform", seed=2)
    b = m.matvec(xt)
    db = torch.from_numpy(b).cuda()
    dx = torch.empty_like(db)
    plan.set_schedule(variant=S._lib.VAR_WAVE, block_warps=2)
    plan.solve_f64(db, dx)
    S.sync_status()
    assert O.rel_err(dx.cpu().numpy(), O.solve(m.rowptr, m.colidx, m.val, b)) <= TOL
    plan.close()
    S.free_device_analysis(L, info)


def test_selector_skips_classes_that_do_not_apply(torch_cuda):
    """A network that ranks a WAVE class first: on a grid it is taken, on a
    banded matrix the next class in predicted order is."""
    import sptrsv_b200 as S
    from sptrsv_b200 import select as SEL

    net = SEL.Mlp(seed=1)
    p = np.zeros(SEL.N_PARAMS, np.float32)
    b3 = np.arange(SEL.N_CLASSES, dtype=np.float32)
    b3[2] = -10.0  # a WAVE class first, then class 0, 1, 3, ...
    p[-SEL.N_CLASSES:] = b3
    net.set_params(p)
    net.set_normalization(np.zeros(SEL.N_FEATURES, np.float32), np.ones(SEL.N_FEATURES, np.float32))
    for m, want in ((gen.grid2d(96, 64, seed=1), 2), (gen.banded(4000, 64, 4, 8, seed=1), 0)):
        L, info = _setup(S, m, S.MULTIROW)
        plan = S.Plan(L, info)
        assert net.select(plan, L, info) == want
        assert plan.schedule().variant == SEL.schedule_from_class(want).variant
        plan.close()
        S.free_device_analysis(L, info)
    net.close()


def test_strip_full_size_grid(torch_cuda):
    import sptrsv_b200 as S

    torch = torch_cuda
    m, xt, k = gen.config("c1")
    b = m.matvec(xt, k)
    ref = O.solve(m.rowptr, m.colidx, m.val, b)
    L, info = _setup(S, m, S.MULTIROW)
    plan = S.Plan(L, info)
    db = torch.from_numpy(b).cuda()
    dx = torch.empty(m.n, dtype=torch.float64, device="cuda")
    scheds = [dict(variant=S._lib.VAR_STRIP, rows_per_warp=r, block_warps=2 if r == 32 else 4) for r in (1, 4, 32)]
    scheds += [dict(variant=S._lib.VAR_WAVE, block_warps=g) for g in (4, 8)]
    for sc in scheds:
        plan.set_schedule(**sc)
        plan.solve_f64(db, dx)
        S.sync_status()
        assert O.rel_err(dx.cpu().numpy(), ref) <= TOL, sc
    plan.close()
    S.free_device_analysis(L, info)


@pytest.mark.parametrize("shape", [(512, 600), (100, 77)], ids=["three_segments", "small"])
def test_streamed_host_solve(torch_cuda, shape):
    """Host-buffer solves of a WAVE plan with pinned b and x copy b in
    segments while the solve runs and write x to the host as line groups finish: the
    result matches the oracle call after call (the segment flags' epochs wrap
    after 255 calls, and b changes between calls), and pageable buffers take
    the plain copy path."""
    import sptrsv_b200 as S

    torch = torch_cuda
    m = gen.grid2d(*shape, seed=3)
    xt = gen.vector(m.n, "uniform", seed=4)
    b = m.matvec(xt)
    ref = O.solve(m.rowptr, m.colidx, m.val, b)
    L, info = _setup(S, m, S.MULTIROW)
    plan = S.Plan(L, info)
    plan.set_schedule(variant=S._lib.VAR_WAVE, block_warps=4)
    hb = torch.from_numpy(b).pin_memory()
    hx = torch.empty(m.n, dtype=torch.float64).pin_memory()
    reps = 260 if m.n < 100_000 else 6
    for r in range(reps):
        scale = 1.0 + r % 3
        hb.copy_(torch.from_numpy(b * scale))
        hx.fill_(float("nan"))
        plan.solve_host(hb, hx, 1, 64)
        assert O.rel_err(hx.numpy(), ref * scale) <= TOL, r
    xp = np.zeros(m.n)
    plan.solve_host(b, xp, 1, 64)
    assert O.rel_err(xp, ref) <= TOL
    plan.solve_host(hb, hx, 1, 32)  # FP32 + refinement: the plain copy path
    assert O.rel_err(hx.numpy(), ref * (1.0 + (reps - 1) % 3)) <= TOL
    plan.close()
    S.free_device_analysis(L, info)


def test_wave_group_of_exactly_48k_shared_memory(torch_cuda):
    """4 lines of 1536 rows per CTA: the FP64 WAVE kernel asks for exactly
    48 KB of dynamic shared memory beside its static shared word, which needs
    the large-shared-memory opt-in (a launch without it is refused)."""
    import sptrsv_b200 as S

    torch = torch_cuda
    m = gen.grid2d(1536, 8, seed=3)
    xt = gen.vector(m.n, "uniform", seed=4)
    b = m.matvec(xt)
    ref = O.solve(m.rowptr, m.colidx, m.val, b)
    L, info = _setup(S, m, S.MULTIROW)
    plan = S.Plan(L, info)
    db = torch.from_numpy(b).cuda()
    dx = torch.empty(m.n, dtype=torch.float64, device="cuda")
    plan.set_schedule(variant=S._lib.VAR_WAVE, block_warps=4, ir_max_iters=2)
    plan.solve_f64(db, dx)
    S.sync_status()
    assert O.rel_err(dx.cpu().numpy(), ref) <= TOL
    plan.solve_ir(db, dx)
    S.sync_status()
    assert O.rel_err(dx.cpu().numpy(), ref) <= TOL
    plan.close()
    S.free_device_analysis(L, info)
