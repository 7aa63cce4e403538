"""Batched solves (many systems, 1-32 right-hand sides each, one persistent
launch, CUDA-graph replay) against the CPU oracle, system by system."""
import numpy as np
import pytest

from oracle import oracle as O
from sptrsv_b200 import gen

pytestmark = pytest.mark.gpu

TOL = 1e-12


def _make(S, nsys, seed, n_hi=6000):
    mats, ks, xs = gen.batch_config(nsys, seed=seed, n_lo=50, n_hi=n_hi, bw_lo=4, bw_hi=600)
    dev = [S.allocate_memory(m.rowptr, m.colidx, m.val, m.n) for m in mats]
    bs = [m.matvec(x, k) for m, x, k in zip(mats, xs, ks)]
    refs = [O.solve(m.rowptr, m.colidx, m.val, b, nrhs=k) for m, b, k in zip(mats, bs, ks)]
    return mats, ks, xs, dev, bs, refs


@pytest.mark.parametrize("precision", [64, 32])
def test_batch_matches_oracle_per_system(torch_cuda, precision):
    import sptrsv_b200 as S
    from sptrsv_b200.batch import Batch

    torch = torch_cuda
    mats, ks, xs, dev, bs, refs = _make(S, 24, seed=5)
    batch = Batch(dev, ks)
    assert batch.vec_len == sum(m.n * k for m, k in zip(mats, ks))
    assert np.array_equal(np.diff(batch.offsets), [m.n * k for m, k in zip(mats, ks)])
    db = torch.from_numpy(np.concatenate(bs)).cuda()
    dx = torch.empty_like(db)
    for sched, width in ((dict(), None), (dict(mode=1, block_warps=4, warps_per_sm=16), None), (dict(mode=0), None),
                         (dict(mode=0, block_warps=4, warps_per_sm=16), None),
                         (dict(mode=0, block_warps=16, backoff_ns=100), None),
                         (dict(mode=2), 16.0), (dict(mode=2, block_warps=4), 1e9), (dict(mode=2, block_warps=2), 4.0),
                         (dict(mode=2, block_warps=16), 0.0)):
        if width is not None:
            batch.set_seq_width(width)
        batch.set_schedule(**sched)
        if width == 1e9:
            assert batch.seq_systems()[0] == len(mats) and batch.seq_systems()[2] == 0
        if width == 0.0:
            assert batch.seq_systems() == (0, 0, batch.n)
        batch.solve(db, dx, precision)
        S.sync_status()
        xh = dx.cpu().numpy()
        for s in range(len(mats)):
            a, b = batch.offsets[s], batch.offsets[s + 1]
            assert O.rel_err(xh[a:b], refs[s]) <= TOL, (s, sched, width)
    batch.close()
    for d in dev:
        S.free_device_analysis(d, None)


def test_batch_graph_replay(torch_cuda):
    import sptrsv_b200 as S
    from sptrsv_b200.batch import Batch

    torch = torch_cuda
    mats, ks, xs, dev, bs, refs = _make(S, 12, seed=6)
    batch = Batch(dev, ks)
    db = torch.from_numpy(np.concatenate(bs)).cuda()
    dx = torch.empty_like(db)
    for rep in range(3):
        dx.fill_(0)
        batch.solve_graph(db, dx, 32)
        S.sync_status()
        xh = dx.cpu().numpy()
        for s in range(len(mats)):
            a, b = batch.offsets[s], batch.offsets[s + 1]
            assert O.rel_err(xh[a:b], refs[s]) <= TOL, (rep, s)
    # a new right-hand side through the same graph (b is read at replay time)
    bs2 = [m.matvec(2.0 * x, k) for m, x, k in zip(mats, xs, ks)]
    db.copy_(torch.from_numpy(np.concatenate(bs2)))
    batch.solve_graph(db, dx, 32)
    S.sync_status()
    xh = dx.cpu().numpy()
    for s in range(len(mats)):
        a, b = batch.offsets[s], batch.offsets[s + 1]
        assert O.rel_err(xh[a:b], 2.0 * refs[s]) <= TOL
    batch.close()
    for d in dev:
        S.free_device_analysis(d, None)


def test_batch_unit_values_exact(torch_cuda):
    import sptrsv_b200 as S
    from sptrsv_b200.batch import Batch

    torch = torch_cuda
    mats, ks, _, _, _, _ = _make(S, 8, seed=7, n_hi=2000)
    units = [m.unit_values() for m in mats]
    dev = [S.allocate_memory(m.rowptr, m.colidx, m.val, m.n) for m in units]
    batch = Batch(dev, ks)
    b = np.concatenate([np.repeat(np.diff(m.rowptr).astype(np.float64), k) for m, k in zip(units, ks)])
    db = torch.from_numpy(b).cuda()
    dx = torch.empty_like(db)
    batch.set_seq_width(1e9)
    for mode in (0, 1, 2):
        batch.set_schedule(mode=mode, block_warps=4)
        for prec in (64, 32):
            batch.solve(db, dx, prec)
            S.sync_status()
            assert bool((dx == 1.0).all()), (mode, prec)
    batch.close()
    for d in dev:
        S.free_device_analysis(d, None)


@pytest.mark.parametrize("precision", [64, 32])
def test_batch_hybrid_many_systems_per_warp(torch_cuda, precision):
    """More near-chain systems than sequential warps: each warp walks several
    systems one after another (one block of two warps per SM)."""
    import sptrsv_b200 as S
    from sptrsv_b200.batch import Batch

    torch = torch_cuda
    mats, ks, xs = gen.batch_config(400, seed=11, n_lo=40, n_hi=300, bw_lo=2, bw_hi=40)
    dev = [S.allocate_memory(m.rowptr, m.colidx, m.val, m.n) for m in mats]
    bs = [m.matvec(x, k) for m, x, k in zip(mats, xs, ks)]
    refs = [O.solve(m.rowptr, m.colidx, m.val, b, nrhs=k) for m, b, k in zip(mats, bs, ks)]
    batch = Batch(dev, ks)
    batch.set_seq_width(1e9)
    batch.set_schedule(mode=2, block_warps=2, warps_per_sm=2)
    nseq, nw, nlvl = batch.seq_systems()
    assert nseq == len(mats) and nlvl == 0 and 0 < nw < nseq
    db = torch.from_numpy(np.concatenate(bs)).cuda()
    dx = torch.empty_like(db)
    for rep in range(2):
        batch.solve_graph(db, dx, precision)
        S.sync_status()
        xh = dx.cpu().numpy()
        for s in range(len(mats)):
            a, b = batch.offsets[s], batch.offsets[s + 1]
            assert O.rel_err(xh[a:b], refs[s]) <= TOL, (rep, s)
    batch.close()
    for d in dev:
        S.free_device_analysis(d, None)


@pytest.mark.parametrize("precision", [64, 32])
def test_batch_long_chains_one_warp_per_rhs(torch_cuda, precision):
    """Long near-chain systems with several right-hand sides are solved by one
    warp per right-hand side (strided columns of b and x): more sequential
    warps than systems, results as the oracle's."""
    import sptrsv_b200 as S
    from sptrsv_b200.batch import Batch

    torch = torch_cuda
    mats, ks, xs = gen.batch_config(6, seed=13, n_lo=20000, n_hi=40000, bw_lo=8, bw_hi=20, k_max=9)
    dev = [S.allocate_memory(m.rowptr, m.colidx, m.val, m.n) for m in mats]
    bs = [m.matvec(x, k) for m, x, k in zip(mats, xs, ks)]
    refs = [O.solve(m.rowptr, m.colidx, m.val, b, nrhs=k) for m, b, k in zip(mats, bs, ks)]
    batch = Batch(dev, ks)
    batch.set_seq_width(16.0)
    batch.set_schedule(mode=2, block_warps=8, ir_iters=2)
    nseq, nw, _ = batch.seq_systems()
    assert nseq == len(mats) and nw > nseq, (nseq, nw, ks)
    db = torch.from_numpy(np.concatenate(bs)).cuda()
    dx = torch.empty_like(db)
    for rep in range(2):
        batch.solve(db, dx, precision)
        S.sync_status()
        xh = dx.cpu().numpy()
        for s in range(len(mats)):
            a, b = batch.offsets[s], batch.offsets[s + 1]
            assert O.rel_err(xh[a:b], refs[s]) <= TOL, (rep, s)
    batch.close()
    for d in dev:
        S.free_device_analysis(d, None)


def test_full_c3_batch_fp64_and_ir_graph(torch_cuda):
    """The full batched configuration: 512 banded systems, n log-uniform in
    [1e3, 2e5], bandwidth log-uniform in [16, 4096], 4-16 off-diagonals per
    row, 1-32 right-hand sides each (2.4e9-byte packed vectors, int64
    packed offsets).  FP64 and FP32 + FP64 refinement through the CUDA
    graph, replayed twice, every system against the oracle; then the hybrid
    split with more systems on sequential warps, where systems with many
    right-hand sides are cut into one unit per column."""
    import sptrsv_b200 as S
    from sptrsv_b200.batch import Batch

    torch = torch_cuda
    mats, ks, xs = gen.batch_config(512, seed=3)
    dev = [S.allocate_memory(m.rowptr, m.colidx, m.val, m.n) for m in mats]
    bs = [m.matvec(x, k) for m, x, k in zip(mats, xs, ks)]
    batch = Batch(dev, ks)
    # the packed vectors hold 2.37 GB each (offsets past 2^31 bytes)
    assert batch.vec_len == sum(m.n * k for m, k in zip(mats, ks)) and batch.vec_len * 8 > 2**31
    refs = [O.solve(m.rowptr, m.colidx, m.val, b, nrhs=k) for m, b, k in zip(mats, bs, ks)]  # about 2 s
    db = torch.from_numpy(np.concatenate(bs)).cuda()
    del bs
    dx = torch.empty_like(db)

    def check(tag):
        xh = dx.cpu().numpy()
        worst = 0.0
        for s in range(len(mats)):
            a, b = batch.offsets[s], batch.offsets[s + 1]
            worst = max(worst, O.rel_err(xh[a:b], refs[s]))
        assert worst <= TOL, (tag, worst)
        return worst

    for part, sched, width, prec, iters in ((0, dict(mode=2, block_warps=4), 16.0, 64, 0),
                                            (0, dict(mode=2, block_warps=4), 16.0, 32, 1),
                                            (0, dict(mode=2, block_warps=8), 64.0, 64, 0),
                                            (4096, dict(mode=2, block_warps=4), 16.0, 64, 0),
                                            (4096, dict(mode=2, block_warps=4), 16.0, 32, 1)):
        batch.set_partition(part)
        batch.set_seq_width(width)
        batch.set_schedule(ir_iters=iters, **sched)
        for rep in range(2):
            dx.fill_(0)
            batch.solve_graph(db, dx, prec)
            S.sync_status()
            check((sched, width, prec, rep))
    nseq, nseqw, _ = batch.seq_systems()  # of the block systems (a warp may take several)
    assert nseq > 0 and nseqw > 0
    batch.close()
    for d in dev:
        S.free_device_analysis(d, None)


@pytest.mark.parametrize("block_rows", [256, 1500])
def test_batch_partitioned(torch_cuda, block_rows):
    """Long systems cut into blocks with warm-ups, solved as a batch of block
    systems; FP64 and FP32 + refinement, plain and graph solves, against the
    oracle; then back to the plain batch."""
    import sptrsv_b200 as S
    from sptrsv_b200.batch import Batch

    torch = torch_cuda
    mats, ks, xs, dev, bs, refs = _make(S, 40, seed=17, n_hi=20000)
    batch = Batch(dev, ks)
    db = torch.from_numpy(np.concatenate(bs)).cuda()
    dx = torch.empty_like(db)
    batch.set_partition(block_rows)
    pi = batch.partition_info()
    long_sys = sum(1 for m in mats if m.n >= 2 * block_rows)
    assert 0 < pi["systems_cut"] <= long_sys and pi["inner_systems"] > len(mats)
    assert pi["warm_rows"] > 0 and 0.0 <= pi["bound"] <= 2.0 ** -60
    for sched, width in ((dict(mode=2, block_warps=4), 16.0), (dict(mode=0), 16.0), (dict(mode=2), 1e9)):
        batch.set_seq_width(width)
        for prec, iters in ((64, 0), (32, 2)):
            batch.set_schedule(ir_iters=iters, **sched)
            for solve in (batch.solve, batch.solve_graph):
                dx.fill_(0)
                solve(db, dx, prec)
                S.sync_status()
                xh = dx.cpu().numpy()
                for s in range(len(mats)):
                    a, b = batch.offsets[s], batch.offsets[s + 1]
                    assert O.rel_err(xh[a:b], refs[s]) <= TOL, (s, sched, prec)
    batch.set_partition(0)
    assert batch.partition_info()["systems_cut"] == 0
    batch.solve(db, dx, 64)
    S.sync_status()
    xh = dx.cpu().numpy()
    for s in range(len(mats)):
        a, b = batch.offsets[s], batch.offsets[s + 1]
        assert O.rel_err(xh[a:b], refs[s]) <= TOL
    batch.close()
    for d in dev:
        S.free_device_analysis(d, None)
