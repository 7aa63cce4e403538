"""The warm-up search of the partitioned solve, on the host (no GPU): for
every block the library picks, solving the block alone from its warm-up
start with a zero boundary reproduces the block's rows of the exact solution
to within rounding — the dropped rows' effect is below the 2^-60 bound the
library reports — while a much shorter warm-up does not.  The solutions here
come from scipy's triangular solve, independent of the library."""
import ctypes

import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as sla

from sptrsv_b200 import _lib as C
from sptrsv_b200 import gen


def _blocks(m, P):
    h = C.HostCsr(m.n, m.nnz, m.rowptr.ctypes.data_as(C.POINTER(C.c_int)),
                  m.colidx.ctypes.data_as(C.POINTER(C.c_int)), m.val.ctypes.data_as(C.POINTER(C.c_double)))
    tab = np.zeros(4 * P, dtype=np.int32)
    bound = ctypes.c_double(0)
    C.check(C.lib().sptrsv_partition_blocks_host(ctypes.byref(h), P, tab.ctypes.data, ctypes.byref(bound)))
    return tab.reshape(P, 4), bound.value


def _block_solution(A, b, s, e):
    """Rows [s, e) solved alone, every entry before s dropped (zero boundary)."""
    return sla.spsolve_triangular(A[s:e, s:e].tocsr(), b[s:e], lower=True)


CASES = {
    "banded_random_signs": (lambda: gen.banded(30000, 256, 8, 8, seed=0), 16),
    "banded_narrow": (lambda: gen.banded(40000, 16, 4, 16, seed=11), 32),
    "grid2d": (lambda: gen.grid2d(300, 200, seed=1), 8),
    "grid3d": (lambda: gen.grid3d(30, 30, 30, seed=3), 6),
    "chain": (lambda: gen.banded(20000, 1, 1, 1, seed=2), 16),
}


@pytest.mark.parametrize("name", list(CASES))
def test_warmups_reproduce_the_exact_rows(name):
    make, P = CASES[name]
    m = make()
    A = sp.csr_matrix((m.val, m.colidx, m.rowptr), shape=(m.n, m.n))
    x = gen.vector(m.n, "uniform", seed=5)
    b = A @ x
    xs = sla.spsolve_triangular(A, b, lower=True)
    tab, bound = _blocks(m, P)
    assert 0.0 <= bound <= 2.0 ** -60
    s, a, e, base = tab.T
    assert a[0] == 0 and e[-1] == m.n and np.all(e[:-1] == a[1:]) and np.all(s <= a)
    assert np.array_equal(base, np.concatenate([[0], np.cumsum(e - s)[:-1]]))
    scale = np.abs(xs).max()
    cut_somewhere = False
    for i in range(P):
        z = _block_solution(A, b, s[i], e[i])
        err = np.abs(z[a[i] - s[i]:] - xs[a[i]:e[i]]).max() / scale
        assert err <= 1e-13, (i, err)  # rounding only: the dropped rows weigh < 2^-60
        if i > 0 and a[i] - s[i] >= 16:
            # a warm-up a quarter as long leaves the boundary's effect visible
            s_short = a[i] - (a[i] - s[i]) // 4
            z = _block_solution(A, b, s_short, e[i])
            err_short = np.abs(z[a[i] - s_short:] - xs[a[i]:e[i]]).max() / scale
            cut_somewhere |= err_short > 1e-10
    assert cut_somewhere


def test_refuses_a_matrix_that_is_not_diagonally_dominant():
    m = gen.banded(20000, 64, 4, 8, seed=1).unit_values()
    with pytest.raises(C.SptrsvError) as ei:
        _blocks(m, 4)
    assert ei.value.code == -9
