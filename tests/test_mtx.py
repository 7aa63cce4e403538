"""MatrixMarket ingest and lower-triangle extraction (the reference driver's
main.cu:66-246 path), checked against a dense numpy computation."""
import numpy as np
import pytest

from sptrsv_b200 import SptrsvError, check_csr_host, gen


def _write(path, banner, n, entries, comments=("% a comment",)):
    lines = [banner] + list(comments) + [f"{n} {n} {len(entries)}"]
    for e in entries:
        lines.append(" ".join(str(v) for v in e))
    path.write_text("\n".join(lines) + "\n")


def _dense_lower(n, entries, symmetric=False, skew=False, pattern=False):
    A = np.zeros((n, n))
    for e in entries:
        i, j = e[0] - 1, e[1] - 1
        v = 1.0 if pattern else float(e[2])
        A[i, j] += v
        if (symmetric or skew) and i != j:
            A[j, i] += -v if skew else v
    return np.tril(A)


def _to_dense(m):
    D = np.zeros((m.n, m.n))
    for i in range(m.n):
        for p in range(m.rowptr[i], m.rowptr[i + 1]):
            D[i, m.colidx[p]] = m.val[p]
    return D


def test_general_unsorted_duplicates_and_missing_diagonal(tmp_path):
    rng = np.random.default_rng(0)
    n = 40
    entries = [(int(i), int(j), round(float(v), 6)) for i, j, v in
               zip(rng.integers(1, n + 1, 300), rng.integers(1, n + 1, 300), rng.uniform(-2, 2, 300))]
    entries += [(3, 3, 2.5), (3, 3, 0.5)]  # duplicate diagonal
    p = tmp_path / "g.mtx"
    _write(p, "%%MatrixMarket matrix coordinate real general", n, entries)
    m = gen.read_mtx_lower(p, unit_values=False)
    assert check_csr_host(m.rowptr, m.colidx) == -1  # sorted, diagonal last
    D = _dense_lower(n, entries)
    missing = np.diag(D) == 0
    D[np.diag_indices(n)] = np.where(missing & ~np.isin(np.arange(n), [e[0] - 1 for e in entries if e[0] == e[1]]),
                                     1.0, np.diag(D))
    got = _to_dense(m)
    off = ~np.eye(n, dtype=bool)
    assert np.allclose(got[off], D[off])
    for i in range(n):
        had = any(e[0] == e[1] == i + 1 for e in entries)
        assert got[i, i] == (D[i, i] if had else 1.0)


@pytest.mark.parametrize("kind", ["symmetric", "skew-symmetric"])
def test_symmetric_expansion(tmp_path, kind):
    n = 6
    entries = [(1, 1, 4.0), (2, 1, -1.0), (3, 2, 2.0), (6, 1, 0.5), (5, 5, 3.0), (6, 4, 1.5)]
    if kind == "skew-symmetric":
        entries = [e for e in entries if e[0] != e[1]]
    p = tmp_path / "s.mtx"
    _write(p, f"%%MatrixMarket matrix coordinate real {kind}", n, entries)
    m = gen.read_mtx_lower(p, unit_values=False)
    D = _dense_lower(n, entries, symmetric=kind == "symmetric", skew=kind == "skew-symmetric")
    got = _to_dense(m)
    off = ~np.eye(n, dtype=bool)
    assert np.allclose(got[off], D[off])


def test_pattern_and_reference_unit_values(tmp_path):
    # the reference forces every value to 1.0 (main.cu:228,236); its test then
    # solves with b = row sums and expects x == 1 exactly
    n = 30
    rng = np.random.default_rng(1)
    entries = sorted({(int(i), int(j)) for i, j in zip(rng.integers(1, n + 1, 120), rng.integers(1, n + 1, 120))})
    p = tmp_path / "p.mtx"
    _write(p, "%%MatrixMarket matrix coordinate pattern general", n, entries)
    m = gen.read_mtx_lower(p, unit_values=True)
    assert np.all(m.val == 1.0)
    D = _dense_lower(n, entries, pattern=True) != 0
    D[np.diag_indices(n)] = True
    assert np.array_equal(_to_dense(m) != 0, D)
    from oracle import oracle as O

    x = O.solve(m.rowptr, m.colidx, m.val, np.diff(m.rowptr).astype(np.float64))
    assert np.all(x == 1.0)


def test_rejects_bad_files(tmp_path):
    p = tmp_path / "bad.mtx"
    p.write_text("%%MatrixMarket matrix array real general\n2 2\n1\n2\n3\n4\n")
    with pytest.raises(SptrsvError):
        gen.read_mtx_lower(p)
    p.write_text("%%MatrixMarket matrix coordinate real general\n2 3 1\n1 1 1.0\n")
    with pytest.raises(SptrsvError):
        gen.read_mtx_lower(p)
    with pytest.raises(SptrsvError):
        gen.read_mtx_lower(tmp_path / "missing.mtx")
