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


def test_long_lines_and_an_inflated_entry_count(tmp_path):
    p = tmp_path / "long.mtx"
    # a comment longer than any fixed line buffer is still one comment
    _write(p, "%%MatrixMarket matrix coordinate real general", 3, [(1, 1, 2.0), (2, 1, -1.0), (2, 2, 4.0), (3, 3, 5.0)],
           comments=("%" + "x" * 20000,))
    m = gen.read_mtx_lower(p, unit_values=False)
    assert m.n == 3 and np.allclose(_to_dense(m), [[2, 0, 0], [-1, 4, 0], [0, 0, 5]])
    # a size line claiming far more entries than the file holds is refused, not allocated for
    p.write_text("%%MatrixMarket matrix coordinate real general\n3 3 999999999999\n1 1 1.0\n")
    with pytest.raises(SptrsvError):
        gen.read_mtx_lower(p)


_FUZZ = r"""
import ctypes, json, sys
import numpy as np
from sptrsv_b200 import _lib as C
rng = np.random.default_rng(7)
d = sys.argv[1]
tokens = ["%%MatrixMarket", "matrix", "coordinate", "real", "pattern", "integer", "general", "symmetric",
          "skew-symmetric", "%", "1", "2", "3", "0", "-1", "4", "1e300", "nan", "x", "", "\t", "99999999999"]
codes = []
for t in range(300):
    if t % 3 == 0:  # a valid file, then perhaps one line replaced by shuffled tokens
        n = int(rng.integers(1, 6))
        ent = [(int(rng.integers(1, n + 1)), int(rng.integers(1, n + 1)), float(rng.normal())) for _ in range(6)]
        lines = ["%%MatrixMarket matrix coordinate real " + str(rng.choice(["general", "symmetric"])),
                 f"{n} {n} {len(ent)}"] + [f"{i} {j} {v}" for i, j, v in ent]
        if rng.random() < 0.5:
            lines[int(rng.integers(0, len(lines)))] = " ".join(rng.choice(tokens, size=rng.integers(0, 5)))
    else:
        lines = ["%%MatrixMarket matrix coordinate real general" if rng.random() < 0.7 else
                 " ".join(rng.choice(tokens, size=rng.integers(1, 6)))]
        for _ in range(int(rng.integers(0, 8))):
            lines.append(" ".join(rng.choice(tokens, size=rng.integers(0, 5))))
    path = f"{d}/f{t}.mtx"
    data = "\n".join(lines)
    if rng.random() < 0.2:  # raw bytes, NULs included
        data = rng.integers(0, 256, size=int(rng.integers(1, 400)), dtype=np.uint8).tobytes().decode("latin-1")
    open(path, "w", encoding="latin-1").write(data)
    m = C.HostCsr()
    r = C.lib().sptrsv_read_mtx_lower(path.encode(), 0, ctypes.byref(m))
    ok = True
    if r == 0:
        bad = ctypes.c_int(-1)
        ok = C.lib().sptrsv_check_csr_host(m.rowptr, m.colidx, m.n, ctypes.byref(bad)) == 0
        C.lib().sptrsv_host_csr_free(ctypes.byref(m))
    codes.append([int(r), bool(ok)])
print(json.dumps(codes))
"""


def test_garbage_files_give_an_error_or_a_valid_matrix(tmp_path):
    """Seeded random files (plausible lines, shuffled tokens, raw bytes) read in
    a child process: each gives an error code or a lower-triangular CSR with
    the diagonal last, and none crashes the reader."""
    import json
    import subprocess
    import sys

    from conftest import ROOT

    r = subprocess.run([sys.executable, "-c", _FUZZ, str(tmp_path)], cwd=ROOT, capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    codes = json.loads(r.stdout.strip().splitlines()[-1])
    assert len(codes) == 300
    assert all(code in (0, -2, -7, -9) for code, _ in codes)
    assert all(ok for code, ok in codes if code == 0)
    assert any(code == 0 for code, _ in codes) and any(code == -2 for code, _ in codes)
