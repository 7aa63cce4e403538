"""Schedule selection on the GPU: features, autotuner, and the MLP's CUDA
forward/backward/Adam kernels against the CPU oracle."""
import numpy as np
import pytest

from oracle import oracle as O
from sptrsv_b200 import gen

pytestmark = pytest.mark.gpu


def _setup(S, m):
    L = S.allocate_memory(m.rowptr, m.colidx, m.val, m.n)
    info = S.AnalysisInfo()
    info.mode = S.ALL
    assert S.run_analysis(info, L) == 0
    return L, info


def _problem(seed, B):
    rng = np.random.default_rng(seed)
    X = rng.standard_normal((B, 12)).astype(np.float32) * 3 + 1
    T = rng.random((B, 24)).astype(np.float32)
    M = (rng.random((B, 24)) > 0.15).astype(np.float32)
    return X, T, M


def test_mlp_forward_and_gradient_match_oracle(torch_cuda):
    from sptrsv_b200 import select as SEL

    net = SEL.Mlp(seed=3)
    mean = np.linspace(-1, 1, 12).astype(np.float32)
    std = np.linspace(0.5, 2, 12).astype(np.float32)
    net.set_normalization(mean, std)
    X, T, M = _problem(4, 37)
    P = net.params()
    Y = net.forward(X)
    Yo = O.mlp_forward(P, mean, std, X)
    assert np.allclose(Y, Yo, rtol=1e-4, atol=1e-4)
    loss, g = net.gradient(X, T, M)
    lo, go = O.mlp_gradient(P, mean, std, X, T, M)
    assert abs(loss - lo) <= 1e-4 * max(1.0, abs(lo))
    err = np.abs(g - go)
    assert np.all(err <= 1e-5 + 1e-3 * np.abs(go)), float(err.max())
    # gradients are deterministic (no atomics in the reductions)
    _, g2 = net.gradient(X, T, M)
    assert np.array_equal(g, g2)
    net.close()


def test_mlp_training_fits_a_known_selector(torch_cuda):
    from sptrsv_b200 import select as SEL

    rng = np.random.default_rng(7)
    N = 600
    X = rng.standard_normal((N, 12)).astype(np.float32)
    # ground-truth relative times: smooth functions of two features
    centers = rng.standard_normal((24, 2))
    T = np.stack([np.sum((X[:, :2] - c) ** 2, axis=1) for c in centers], axis=1) * 0.3
    T = (T - T.min(axis=1, keepdims=True)).astype(np.float32)
    M = np.ones_like(T)
    net = SEL.Mlp(seed=1)
    net.set_normalization(X.mean(0), X.std(0))
    curve = net.train(X, T, M, epochs=150, batch=64, lr=3e-3, seed=2)
    assert curve[-1] < 0.1 * curve[0]
    pred = net.forward(X).argmin(axis=1)
    regret = T[np.arange(N), pred]
    assert np.mean(pred == T.argmin(axis=1)) > 0.6 and np.mean(regret) < 0.15
    net.close()


def test_features_match_host_computation(torch_cuda):
    import sptrsv_b200 as S
    from sptrsv_b200 import select as SEL

    m = gen.zipf(30000, 1.5, 256, seed=2)
    L, info = _setup(S, m)
    f = SEL.features(L, info)
    a = O.analysis(m.rowptr, m.colidx)
    offs = np.diff(m.rowptr) - 1
    widths = np.bincount(a["levels"] - 1)
    expect = [np.log2(m.n), np.log2(m.nnz), m.nnz / m.n, np.log2(a["nlevs"]), np.log2(m.n / a["nlevs"]),
              np.log2(widths.max())]
    assert np.allclose(f[:6], expect, rtol=1e-5)
    q = np.sort(offs)
    for j, qq in zip(range(6, 10), (0.25, 0.5, 0.9, 0.99)):
        v = q[int(np.ceil(qq * m.n)) - 1]
        assert f[j] == (v if v < 256 else 2.0 ** np.floor(np.log2(v)))
    assert np.isclose(f[10], np.log2(1 + offs.max()))
    assert np.isclose(f[11], np.mean(offs == 0))
    S.free_device_analysis(L, info)


def test_autotune_picks_fastest_and_stays_correct(torch_cuda):
    import sptrsv_b200 as S
    from sptrsv_b200 import select as SEL

    torch = torch_cuda
    m = gen.grid2d(200, 200, seed=1)
    L, info = _setup(S, m)
    plan = S.Plan(L, info)
    b = m.matvec(gen.vector(m.n, "uniform", seed=3))
    db = torch.from_numpy(b).cuda()
    dx = torch.empty_like(db)
    best, times = SEL.autotune(plan, db, dx, 1, 32, reps=2)
    assert np.isfinite(times).sum() == 24
    assert best == int(np.nanargmin(times))
    s = plan.schedule()
    ref_s = SEL.schedule_from_class(best)
    assert (s.variant, s.rows_per_warp, s.band_levels, s.cluster_rows) == \
           (ref_s.variant, ref_s.rows_per_warp, ref_s.band_levels, ref_s.cluster_rows)
    plan.solve_ir(db, dx)
    S.sync_status()
    assert O.rel_err(dx.cpu().numpy(), O.solve(m.rowptr, m.colidx, m.val, b)) <= 1e-12
    # the MLP path sets a schedule from the features
    net = SEL.Mlp(seed=0)
    cls = net.select(plan, L, info)
    assert 0 <= cls < 24
    plan.solve_ir(db, dx)
    S.sync_status()
    assert O.rel_err(dx.cpu().numpy(), O.solve(m.rowptr, m.colidx, m.val, b)) <= 1e-12
    net.close()
    plan.close()
    S.free_device_analysis(L, info)


def test_selector_retrained_on_gpu_and_remeasured_live(torch_cuda):
    """The shipped selector's data retrained from scratch by the CUDA forward,
    backward and Adam kernels reaches a held-out regret close to the stored
    evaluation's; then, on fresh matrices outside the data set, every class is
    timed live and the learned choice is compared with the best class and
    with the reference's own rule (its multirow solver for every matrix)."""
    import json
    from pathlib import Path

    import sptrsv_b200 as S
    from sptrsv_b200 import select as SEL
    from sptrsv_b200 import train_selector as TS

    torch = torch_cuda
    pkg = Path(SEL.__file__).resolve().parent
    if not (pkg / "selector_weights.npz").exists():
        pytest.skip("selector not trained")
    d = np.load(pkg / "selector_data.npz")
    ev = json.loads((pkg / "selector_eval.json").read_text())
    X, Tm = d["features"], d["times"]
    ntr = ev["n_train"]
    T, M = SEL.targets_from_times(Tm)
    net = SEL.Mlp(seed=11)
    mean, std = X[:ntr].mean(0), X[:ntr].std(0)
    net.set_normalization(mean, np.where(std > 1e-6, std, 1.0).astype(np.float32))
    curve = net.train(X[:ntr], T[:ntr], M[:ntr], epochs=400, batch=64, lr=2e-3, seed=11)
    assert curve[-1] < 0.5 * curve[0]
    Y = net.forward(X[ntr:])
    Y[~np.isfinite(Tm[ntr:])] = np.inf
    held_out = TS.evaluate(Tm[ntr:], Y.argmin(axis=1))
    assert held_out["mean_regret"] <= ev["mlp"]["test"]["mean_regret"] + 0.10, held_out
    assert held_out["geomean_time_over_best"] <= 1.1, held_out
    net.close()
    # live: fresh matrices (seeds and sizes not in the data set), every class timed
    shipped = SEL.Mlp.load(pkg / "selector_weights.npz")
    ratios_best, ratios_ref = [], []
    for m in (gen.banded(60000, 96, 4, 12, seed=901), gen.grid2d(320, 260, seed=902), gen.grid3d(36, 36, 36, seed=903),
              gen.zipf(80000, 1.5, 256, seed=904)):
        L, info = _setup(S, m)
        plan = S.Plan(L, info)
        b = torch.from_numpy(m.matvec(gen.vector(m.n, "uniform", seed=905))).cuda()
        x = torch.empty_like(b)
        _, times = SEL.autotune(plan, b, x, 1, 64, reps=3)
        cls = shipped.select(plan, L, info)
        plan.solve_f64(b, x)
        S.sync_status()
        assert O.rel_err(x.cpu().numpy(), O.solve(m.rowptr, m.colidx, m.val, b.cpu().numpy())) <= 1e-12
        ratios_best.append(float(times[cls] / np.nanmin(times)))
        ratios_ref.append(float(times[12] / times[cls]))
        plan.close()
        S.free_device_analysis(L, info)
    shipped.close()
    gm = lambda v: float(np.exp(np.mean(np.log(v))))  # noqa: E731
    # the learned choice is close to the exhaustive autotuner's and ahead of the reference's rule
    assert gm(ratios_best) <= 1.5, ratios_best
    assert gm(ratios_ref) >= 1.1, ratios_ref
