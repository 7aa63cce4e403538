"""Train and evaluate the learned schedule selector.

1. Dataset: seeded matrices from five generator families (banded, 2D and
   3D 5/7-point Laplacian lower triangles, Zipf DAGs, block-diagonal with
   dense 32x32 lower blocks), n log-uniform in [n_lo, n_hi].  For each: the
   analysis, the 12 features, and the exhaustive autotuner's median time of
   every one of the 24 schedule classes (FP64 solves, L2 flushed).
2. Training: the MLP 12 -> 64 -> 64 -> 24 regresses log2(time / best time)
   per class (masked MSE, Adam) with the library's CUDA kernels.
3. Evaluation on held-out matrices: regret = time(chosen) / time(best) - 1
   for the MLP, for the best single fixed class, and for the reference's own
   rule (its multirow solver, class 12), plus top-1 accuracy.

Usage (GPU):  python -m sptrsv_b200.train_selector --n-train 2000 --n-test 400 --out sptrsv_b200/selector
Writes <out>_data.npz (features, times, family, n), <out>_weights.npz and
<out>_eval.json.  The dataset can be collected in pieces (--collect-only
--start S --count C --out <piece>, then --data <piece1>,<piece2>,... to
train on their concatenation in matrix order).
"""
from __future__ import annotations

import argparse
import json
import math
import time
from concurrent.futures import ThreadPoolExecutor

import numpy as np

FAMILIES = ["banded", "grid2d", "grid3d", "zipf", "blockdiag"]
REFERENCE_CLASS = 12  # MULTIROW, default preset: the reference's multirow solver


def make_matrix(idx: int, seed: int, n_lo: int, n_hi: int):
    from . import gen

    rng = np.random.default_rng(seed * 7919 + idx)
    fam = FAMILIES[idx % len(FAMILIES)]
    n = int(math.exp(rng.uniform(math.log(n_lo), math.log(n_hi))))
    s = seed * 100_003 + idx
    if fam == "banded":
        bw = int(math.exp(rng.uniform(math.log(16), math.log(4096))))
        lo = int(rng.integers(1, 9))
        m = gen.banded(n, bw, lo, lo + int(rng.integers(0, 9)), seed=s)
    elif fam == "grid2d":
        side = max(8, int(math.sqrt(n)))
        aspect = float(rng.uniform(0.5, 2.0))
        m = gen.grid2d(max(4, int(side * aspect)), max(4, int(side / aspect)), seed=s)
    elif fam == "grid3d":
        side = max(4, int(round(n ** (1 / 3))))
        m = gen.grid3d(side, side, max(4, int(n / side / side)), seed=s)
    elif fam == "zipf":
        m = gen.zipf(n, float(rng.choice([1.3, 1.5, 2.0])), 256, seed=s)
    else:
        m = gen.blockdiag(n, 32, seed=s)
    return fam, m


def collect(n_total: int, seed: int, n_lo: int, n_hi: int, reps: int, log=print, start: int = 0, save=None):
    """Matrices start .. start + n_total - 1 of the seeded sequence.  save(X,
    T, fam, n), when given, is called every 25 matrices with what is done."""
    import torch

    import sptrsv_b200 as S
    from . import select as SEL

    feats, times, fams, ns = [], [], [], []
    with ThreadPoolExecutor(max_workers=4) as ex:
        futs = [ex.submit(make_matrix, start + i, seed, n_lo, n_hi) for i in range(min(n_total, 6))]
        t0 = time.time()
        for i in range(n_total):
            fam, m = futs[i].result()
            if i + 6 < n_total:
                futs.append(ex.submit(make_matrix, start + i + 6, seed, n_lo, n_hi))
            L = S.allocate_memory(m.rowptr, m.colidx, m.val, m.n)
            info = S.AnalysisInfo()
            info.mode = S.ALL
            S.run_analysis(info, L)
            f = SEL.features(L, info)
            plan = S.Plan(L, info)
            b = torch.ones(m.n, dtype=torch.float64, device="cuda")
            x = torch.empty_like(b)
            _, t = SEL.autotune(plan, b, x, 1, 64, reps=reps)
            plan.close()
            S.free_device_analysis(L, info)
            feats.append(f)
            times.append(t)
            fams.append(FAMILIES.index(fam))
            ns.append(m.n)
            if (i + 1) % 25 == 0:
                log(f"  {i + 1}/{n_total} matrices ({time.time() - t0:.0f} s)")
                if save:
                    save(np.array(feats, np.float32), np.array(times, np.float32), np.array(fams, np.int32),
                         np.array(ns, np.int64))
    return (np.array(feats, np.float32), np.array(times, np.float32), np.array(fams, np.int32),
            np.array(ns, np.int64))


def evaluate(times: np.ndarray, choice: np.ndarray) -> dict:
    best = np.nanmin(times, axis=1)
    chosen = times[np.arange(times.shape[0]), choice]
    chosen = np.where(np.isfinite(chosen), chosen, np.nanmax(times, axis=1))
    regret = chosen / best - 1.0
    return {"mean_regret": float(regret.mean()), "median_regret": float(np.median(regret)),
            "p90_regret": float(np.quantile(regret, 0.9)),
            "geomean_time_over_best": float(np.exp(np.mean(np.log(chosen / best)))),
            "top1": float(np.mean(choice == np.nanargmin(times, axis=1)))}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n-train", type=int, default=2000)
    ap.add_argument("--n-test", type=int, default=400)
    ap.add_argument("--n-lo", type=int, default=10_000)
    ap.add_argument("--n-hi", type=int, default=4_000_000)
    ap.add_argument("--reps", type=int, default=2)
    ap.add_argument("--epochs", type=int, default=400)
    ap.add_argument("--seed", type=int, default=4)
    ap.add_argument("--out", default="sptrsv_b200/selector")
    ap.add_argument("--data", default=None,
                    help="reuse dataset npz files (comma-separated pieces, concatenated) instead of collecting")
    ap.add_argument("--collect-only", action="store_true", help="collect matrices start .. start+count-1 and stop")
    ap.add_argument("--start", type=int, default=0)
    ap.add_argument("--count", type=int, default=0)
    args = ap.parse_args()

    import torch

    from . import select as SEL

    torch.cuda.set_device(0)
    if args.collect_only:
        print(f"collecting matrices {args.start} .. {args.start + args.count - 1}", flush=True)
        def save(X, Tm, fam, ns):
            np.savez(f"{args.out}_data.npz", features=X, times=Tm, family=fam, n=ns, start=args.start)

        X, Tm, fam, ns = collect(args.count, args.seed, args.n_lo, args.n_hi, args.reps, start=args.start,
                                 save=save)
        save(X, Tm, fam, ns)
        return
    if args.data:
        zs = [np.load(f) for f in args.data.split(",")]
        zs.sort(key=lambda z: int(z["start"]) if "start" in z.files else 0)
        X = np.concatenate([z["features"] for z in zs])
        Tm = np.concatenate([z["times"] for z in zs])
        fam = np.concatenate([z["family"] for z in zs])
        ns = np.concatenate([z["n"] for z in zs])
        np.savez(f"{args.out}_data.npz", features=X, times=Tm, family=fam, n=ns)
    else:
        print(f"collecting {args.n_train + args.n_test} matrices", flush=True)
        X, Tm, fam, ns = collect(args.n_train + args.n_test, args.seed, args.n_lo, args.n_hi, args.reps)
        np.savez(f"{args.out}_data.npz", features=X, times=Tm, family=fam, n=ns)
    ntr = args.n_train
    if X.shape[0] < args.n_train + args.n_test:  # fewer matrices than asked for: 5/6 train, 1/6 held out
        ntr = X.shape[0] * 5 // 6
        print(f"{X.shape[0]} matrices: {ntr} train, {X.shape[0] - ntr} held out", flush=True)
    T, M = SEL.targets_from_times(Tm)
    net = SEL.Mlp(seed=args.seed)
    mean, std = X[:ntr].mean(0), X[:ntr].std(0)
    std = np.where(std > 1e-6, std, 1.0).astype(np.float32)
    net.set_normalization(mean, std)
    curve = net.train(X[:ntr], T[:ntr], M[:ntr], epochs=args.epochs, batch=64, lr=2e-3, seed=args.seed)
    # the selector takes the best predicted class that applies to the matrix
    # (sptrsv_plan_select_schedule skips classes that fail to set on it, the
    # ones the autotuner could not time)
    scores = net.forward(X)
    scores[~np.isfinite(Tm)] = np.inf
    pred = scores.argmin(axis=1)
    test = slice(ntr, X.shape[0])
    # baselines: the best single class on the training set, the reference's rule
    train_reg = np.nanmean(Tm[:ntr] / np.nanmin(Tm[:ntr], axis=1, keepdims=True), axis=0)
    fixed = int(np.nanargmin(train_reg))
    report = {
        "n_train": ntr, "n_test": int(X.shape[0] - ntr), "n_range": [int(ns.min()), int(ns.max())],
        "epochs": args.epochs, "final_train_loss": float(curve[-1]),
        "mlp": {"train": evaluate(Tm[:ntr], pred[:ntr]), "test": evaluate(Tm[test], pred[test])},
        "fixed_best_class": {"class": fixed, "name": SEL.class_name(fixed),
                             "test": evaluate(Tm[test], np.full(Tm[test].shape[0], fixed))},
        "reference_rule": {"class": REFERENCE_CLASS, "name": SEL.class_name(REFERENCE_CLASS),
                           "test": evaluate(Tm[test], np.full(Tm[test].shape[0], REFERENCE_CLASS))},
        "test_speedup_mlp_vs_reference_rule": float(
            np.exp(np.mean(np.log(Tm[test][:, REFERENCE_CLASS] /
                                  Tm[test][np.arange(Tm[test].shape[0]), pred[test]])))),
    }
    net.save(f"{args.out}_weights.npz")
    with open(f"{args.out}_eval.json", "w") as fh:
        json.dump(report, fh, indent=1)
    print(json.dumps(report, indent=1), flush=True)


if __name__ == "__main__":
    main()
