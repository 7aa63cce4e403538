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
