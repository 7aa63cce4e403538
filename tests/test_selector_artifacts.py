"""The shipped selector (weights, normalisation, training data, evaluation)
is self-consistent: the CPU MLP oracle, run on the stored features with the
stored weights, reproduces the held-out regret the training run reported."""
import json

import numpy as np
import pytest

from conftest import ROOT
from oracle import oracle as O

PKG = ROOT / "sptrsv_b200"


@pytest.mark.skipif(not (PKG / "selector_weights.npz").exists(), reason="selector not trained")
def test_selector_reproduces_reported_regret():
    w = np.load(PKG / "selector_weights.npz")
    d = np.load(PKG / "selector_data.npz")
    ev = json.loads((PKG / "selector_eval.json").read_text())
    assert w["params"].shape == (6552,) and d["features"].shape[1] == 12 and d["times"].shape[1] == 24
    ntr = ev["n_train"]
    X, T = d["features"][ntr:], d["times"][ntr:]
    Y = O.mlp_forward(w["params"], w["mean"], w["std"], X)
    Y[~np.isfinite(T)] = np.inf  # classes that do not apply to a matrix are skipped, as the selector does
    choice = Y.argmin(axis=1)
    best = np.nanmin(T, axis=1)
    chosen = T[np.arange(T.shape[0]), choice]
    regret = float(np.mean(chosen / best - 1.0))
    assert abs(regret - ev["mlp"]["test"]["mean_regret"]) < 0.02
    # the learned choice beats the reference's own rule (its multirow solver) on held-out matrices
    ref = T[:, ev["reference_rule"]["class"]]
    assert float(np.exp(np.mean(np.log(ref / chosen)))) > 1.1


def test_targets_and_evaluation_on_a_small_table():
    """The training targets (log2 of time over the best, masked where a class
    did not run) and the evaluation's regret, top-1 and geometric mean, on a
    table small enough to check by hand."""
    from sptrsv_b200 import select as SEL
    from sptrsv_b200 import train_selector as TS

    t = np.full((2, SEL.N_CLASSES), np.nan, dtype=np.float32)
    t[0, :3] = [2.0, 1.0, 4.0]
    t[1, 5], t[1, 7] = 3.0, 6.0
    T, M = SEL.targets_from_times(t)
    assert np.array_equal(M[0, :4], [1, 1, 1, 0]) and M[1].sum() == 2
    assert np.allclose(T[0, :3], [1.0, 0.0, 2.0]) and np.allclose(T[1, [5, 7]], [0.0, 1.0])
    assert np.all(T[M == 0] == 0)
    ev = TS.evaluate(t, np.array([0, 5]))  # 2x the best on the first matrix, the best on the second
    assert np.isclose(ev["mean_regret"], 0.5) and np.isclose(ev["top1"], 0.5)
    assert np.isclose(ev["geomean_time_over_best"], np.sqrt(2.0))
    # a choice that did not run counts as the slowest class that did
    ev = TS.evaluate(t, np.array([1, 0]))
    assert np.isclose(ev["mean_regret"], 0.5) and np.isclose(ev["top1"], 0.5)


def test_class_table_names_and_the_reference_rule():
    """The 24 schedule classes have distinct names; the indexes the stored
    selector data and the evaluation rely on are fixed: class 12 is the
    reference's own rule (its multirow solver, 8-warp blocks, no back-off),
    class 4 WAVE over 16 blocks, class 23 BAND over 128 blocks."""
    from sptrsv_b200 import select as SEL

    names = [SEL.class_name(c) for c in range(SEL.N_CLASSES)]
    assert len(set(names)) == SEL.N_CLASSES
    assert names[12] == "multirow/bw8-bo0-wps0" and names[4] == "wave/G4-P16" and names[23] == "band-P128"
    ev = json.loads((PKG / "selector_eval.json").read_text()) if (PKG / "selector_eval.json").exists() else None
    if ev is not None:
        assert ev["reference_rule"]["class"] == 12 and ev["reference_rule"]["name"] == names[12]
    with pytest.raises(Exception):
        SEL.schedule_from_class(SEL.N_CLASSES)
