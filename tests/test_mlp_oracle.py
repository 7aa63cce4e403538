"""The MLP oracle (oracle/mlp_oracle.c) against central finite differences and
a numpy restatement — the checker the GPU training kernels are held to."""
import numpy as np

from oracle import oracle as O


def _problem(seed=0, B=7):
    rng = np.random.default_rng(seed)
    P = (rng.standard_normal(6552) * 0.2).astype(np.float32)
    mean = rng.standard_normal(12).astype(np.float32)
    std = (0.5 + rng.random(12)).astype(np.float32)
    X = rng.standard_normal((B, 12)).astype(np.float32) * 2
    T = rng.random((B, 24)).astype(np.float32)
    M = (rng.random((B, 24)) > 0.2).astype(np.float32)
    return P, mean, std, X, T, M


def _np_forward(P, mean, std, X):
    W1 = P[:768].reshape(12, 64).astype(np.float64); b1 = P[768:832]
    W2 = P[832:4928].reshape(64, 64).astype(np.float64); b2 = P[4928:4992]
    W3 = P[4992:6528].reshape(64, 24).astype(np.float64); b3 = P[6528:6552]
    xn = (X.astype(np.float64) - mean) / std
    h1 = np.maximum(xn @ W1 + b1, 0)
    h2 = np.maximum(h1 @ W2 + b2, 0)
    return h2 @ W3 + b3


def test_forward_matches_numpy():
    P, mean, std, X, _, _ = _problem()
    assert np.allclose(O.mlp_forward(P, mean, std, X), _np_forward(P, mean, std, X), rtol=1e-12, atol=1e-12)


def test_gradient_matches_finite_differences():
    P, mean, std, X, T, M = _problem(1)
    loss, G = O.mlp_gradient(P, mean, std, X, T, M)
    Y = _np_forward(P, mean, std, X)
    assert np.isclose(loss, float((M * (Y - T) ** 2).sum() / M.sum()), rtol=1e-10)
    rng = np.random.default_rng(5)
    idx = np.concatenate([rng.choice(6552, 60, replace=False), [0, 767, 768, 4991, 6551]])
    for i in idx:
        h = 1e-3
        Pp, Pm = P.astype(np.float64).copy(), P.astype(np.float64).copy()
        Pp[i] += h
        Pm[i] -= h
        # forward in double with perturbed parameters
        fp = float((M * (_np_forward_d(Pp, mean, std, X) - T) ** 2).sum() / M.sum())
        fm = float((M * (_np_forward_d(Pm, mean, std, X) - T) ** 2).sum() / M.sum())
        fd = (fp - fm) / (2 * h)
        assert abs(fd - G[i]) <= 1e-5 + 1e-4 * abs(G[i]), (i, fd, G[i])


def _np_forward_d(P, mean, std, X):
    W1 = P[:768].reshape(12, 64); b1 = P[768:832]
    W2 = P[832:4928].reshape(64, 64); b2 = P[4928:4992]
    W3 = P[4992:6528].reshape(64, 24); b3 = P[6528:6552]
    xn = (X.astype(np.float64) - mean.astype(np.float64)) / std.astype(np.float64)
    h1 = np.maximum(xn @ W1 + b1, 0)
    h2 = np.maximum(h1 @ W2 + b2, 0)
    return h2 @ W3 + b3
