"""Generate the golden fixtures in tests/golden/ from the REFERENCE's own code.

Runs HCL-Fing/SPTRSV's analysis and solve kernels (built from the reference
sources by `make -C oracle ref` into oracle/_ref/libsptrsv_ref.so) on a GPU
and records, per case: the input CSR and right-hand side, the reference's
level array, nlevs, iorder (MULTIROW and ORDER analyses), n_warps,
ibase_row, ivect_size_warp, and the x each reference solver (simple, order,
multirow) returns, for real values and for the reference's own unit-valued
known-answer input (main.cu:228,236; test.cu:10-15).

Usage (on a machine with a GPU and the built oracle/_ref):
    python tests/golden/make_golden.py [outdir]
The committed fixtures were produced on a B200 with this script.  That run
printed, per case, the sizes, whether the CPU oracle's analysis equals the
reference's, the oracle-vs-reference forward error of each reference solver
and whether the unit-value known-answer test came out exact:

    case                  n     nnz    nlevs n_warps analysis  simple   order    multirow  unit KAT
    banded_n2000          2000  15930  364   1189    equal     4.4e-16  5.6e-16  5.6e-16   exact
    banded_c0shape_n5000  5000  44964  352   1411    equal     5.6e-16  5.6e-16  5.6e-16   exact
    grid2d_48x40          1920  5672   87    207     equal     2.2e-16  2.2e-16  2.2e-16   exact
    grid3d_12x11x10       1320  4918   31    177     equal     3.3e-16  3.3e-16  3.3e-16   exact
    zipf_n3000            3000  72635  131   1130    equal     1.9e-15  1.9e-15  1.9e-15   exact
    blockdiag_n1000       1000  16404  32    637     equal     5.6e-16  5.6e-16  5.6e-16   exact
    chain_n700            700   1399   700   700     equal     2.2e-16  2.2e-16  2.2e-16   exact
    diagonal_n333         333   333    1     11      equal     0        0        1.1e-16   exact
    random_n37            37    277    23    34      equal     3.3e-16  3.3e-16  3.3e-16   exact
    single_n1             1     1      1     1       equal     0        0        0         exact
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle import oracle as O  # noqa: E402
from sptrsv_b200 import gen  # noqa: E402


def chain(n: int, seed: int):
    rng = np.random.default_rng(seed)
    rp = np.concatenate([[0, 1], 1 + 2 * np.arange(1, n)]).astype(np.int32)
    ci = np.concatenate([[0]] + [[i - 1, i] for i in range(1, n)]).astype(np.int32)
    va = np.empty(ci.shape[0])
    va[rp[1:] - 1] = 2.0 + rng.random(n)
    off = np.setdiff1d(np.arange(ci.shape[0]), rp[1:] - 1)
    va[off] = rng.uniform(-1, 1, off.shape[0])
    return gen.from_arrays(rp, ci, va)


def diagonal(n: int, seed: int):
    rng = np.random.default_rng(seed)
    return gen.from_arrays(np.arange(n + 1), np.arange(n), 1.0 + rng.random(n))


def random_sparse(n: int, maxk: int, seed: int):
    rng = np.random.default_rng(seed)
    rows, cols, vals = [0], [], []
    for i in range(n):
        k = int(rng.integers(0, min(i, maxk) + 1)) if i else 0
        c = sorted(rng.choice(i, size=k, replace=False).tolist()) if k else []
        v = rng.uniform(-1, 1, k).tolist()
        cols += c + [i]
        vals += v + [1.0 + float(np.abs(v).sum())]
        rows.append(len(cols))
    return gen.from_arrays(rows, cols, vals)


CASES = {
    "banded_n2000": lambda: gen.banded(2000, 64, 2, 12, seed=21),
    "banded_c0shape_n5000": lambda: gen.banded(5000, 256, 8, 8, seed=0),
    "grid2d_48x40": lambda: gen.grid2d(48, 40, seed=22),
    "grid3d_12x11x10": lambda: gen.grid3d(12, 11, 10, seed=23),
    "zipf_n3000": lambda: gen.zipf(3000, 1.5, 256, seed=24),
    "blockdiag_n1000": lambda: gen.blockdiag(1000, 32, seed=25),
    "chain_n700": lambda: chain(700, 26),
    "diagonal_n333": lambda: diagonal(333, 27),
    "random_n37": lambda: random_sparse(37, 20, 28),
    "single_n1": lambda: gen.from_arrays([0, 1], [0], [2.5]),
}


def main(outdir: Path):
    outdir.mkdir(parents=True, exist_ok=True)
    O.ref_lib().ref_set_watchdog_seconds(60.0)
    for name, make in CASES.items():
        m = make()
        xt = gen.vector(m.n, "uniform", seed=1000 + len(name))
        b = m.matvec(xt)
        rec = {"rowptr": m.rowptr, "colidx": m.colidx, "val": m.val, "b": b, "x_true": xt}
        a = O.ref_analysis(m.rowptr, m.colidx, mode=2)
        a1 = O.ref_analysis(m.rowptr, m.colidx, mode=1)
        rec.update({
            "ref_levels": a["levels"], "ref_nlevs": np.int32(a["nlevs"]), "ref_iorder": a["iorder"],
            "ref_n_warps": np.int32(a["n_warps"]), "ref_ibase_row": a["ibase_row"],
            "ref_ivect_size_warp": a["ivect_size_warp"], "ref_iorder_ordermode": a1["iorder"],
        })
        unit = m.unit_values()
        bu = np.diff(m.rowptr).astype(np.float64)
        for v, vn in ((0, "simple"), (1, "order"), (2, "multirow")):
            rec[f"ref_x_{vn}"], _ = O.ref_solve(v, m.rowptr, m.colidx, m.val, b)
            rec[f"ref_x_unit_{vn}"], _ = O.ref_solve(v, unit.rowptr, unit.colidx, unit.val, bu)
        oa = O.analysis(m.rowptr, m.colidx)
        ox = O.solve(m.rowptr, m.colidx, m.val, b)
        same = (oa["nlevs"] == a["nlevs"] and np.array_equal(oa["levels"], a["levels"])
                and np.array_equal(oa["iorder"], a["iorder"]) and np.array_equal(oa["ibase_row"], a["ibase_row"])
                and np.array_equal(oa["ivect_size_warp"], a["ivect_size_warp"]))
        errs = {v: O.rel_err(rec[f"ref_x_{v}"], ox) for v in ("simple", "order", "multirow")}
        unit_ok = all(np.all(rec[f"ref_x_unit_{v}"] == 1.0) for v in ("simple", "order", "multirow"))
        print(f"{name}: n={m.n} nnz={m.nnz} nlevs={a['nlevs']} n_warps={a['n_warps']} "
              f"oracle==ref analysis: {same}; ref-vs-oracle x err: "
              + " ".join(f"{k}={e:.1e}" for k, e in errs.items()) + f"; unit KAT exact: {unit_ok}", flush=True)
        np.savez_compressed(outdir / f"{name}.npz", **rec)


if __name__ == "__main__":
    main(Path(sys.argv[1]) if len(sys.argv) > 1 else Path(__file__).resolve().parent)
