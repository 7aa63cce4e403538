"""The C ABI library loads without a GPU and exports every declared symbol;
host-side checks and generators behave."""
import ctypes
import re

import numpy as np
import pytest

from conftest import ROOT


def _declared_functions():
    text = (ROOT / "include" / "sptrsv_b200.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = set()
    for m in re.finditer(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b([A-Za-z_]\w*)\s*\(", text, flags=re.M):
        name = m.group(1)
        if name not in {"if", "while", "for", "sizeof", "return", "defined"}:
            names.add(name)
    return sorted(names)


def test_library_loads_and_exports_every_declared_symbol():
    import sptrsv_b200

    L = sptrsv_b200.lib()
    decl = _declared_functions()
    assert len(decl) > 30
    missing = [n for n in decl if not hasattr(L, n)]
    assert not missing, f"declared but not exported: {missing}"
    # the reference's entry points keep their exact, unmangled names
    for n in ["allocate_memory", "run_analysis", "run_solver", "free_device_analysis",
              "multirow_analysis_base_GPU", "csr_L_solve_simple", "csr_L_solve_order", "csr_L_solve_multirow"]:
        assert n in decl


def test_python_binding_covers_abi():
    from sptrsv_b200 import _lib

    assert set(_lib.exported_symbols()) == set(_declared_functions())


def test_struct_layouts_match_reference():
    # header/dfr_syncfree.h:14-41 on LP64: field offsets as a C compiler lays them out
    from sptrsv_b200._lib import AnalysisInfo, SpMat

    assert [SpMat.nr.offset, SpMat.nc.offset, SpMat.nnz.offset, SpMat.ia.offset, SpMat.ja.offset, SpMat.a.offset] \
        == [0, 4, 8, 16, 24, 32]
    assert ctypes.sizeof(SpMat) == 40
    assert AnalysisInfo.mode.offset == 0 and AnalysisInfo.nlevs.offset == 8
    assert AnalysisInfo.lev_size.offset == 16 and AnalysisInfo.n_warps.offset == 32
    assert AnalysisInfo.row_ctr.offset == 72 and ctypes.sizeof(AnalysisInfo) == 80


def test_header_compiles_as_c_and_struct_sizes(tmp_path):
    import subprocess

    src = tmp_path / "t.c"
    src.write_text('#include "sptrsv_b200.h"\n#include <stdio.h>\n#include <stddef.h>\n'
                   'int main(void){printf("%zu %zu %zu\\n", sizeof(sp_mat_t), sizeof(dfr_analysis_info_t),'
                   ' offsetof(dfr_analysis_info_t,row_ctr)); return SIMPLE+ORDER+MULTIROW+ALL == 6 ? 0 : 1;}\n')
    exe = tmp_path / "t"
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", f"-I{ROOT / 'include'}", str(src), "-o", str(exe)],
                   check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()
    assert out == ["40", "80", "72"]


def test_check_csr_host_rejects_malformed():
    from sptrsv_b200 import check_csr_host

    good = (np.array([0, 1, 3, 5]), np.array([0, 0, 1, 1, 2]))
    assert check_csr_host(*good) == -1
    assert check_csr_host(np.array([0, 1, 2, 4]), np.array([0, 0, 1, 2])) == 1       # row 1 misses its diagonal
    assert check_csr_host(np.array([0, 1, 3, 5]), np.array([0, 1, 0, 1, 2])) == 1    # diagonal not last
    assert check_csr_host(np.array([0, 1, 3, 6]), np.array([0, 0, 1, 1, 0, 2])) == 2  # unsorted
    assert check_csr_host(np.array([0, 1, 3, 5]), np.array([0, 2, 1, 1, 2])) == 1    # col >= row
    assert check_csr_host(np.array([0, 1, 1, 3]), np.array([0, 1, 2])) == 1          # empty row
    assert check_csr_host(np.array([0]), np.array([], dtype=np.int32)) == -1          # n = 0


def test_allocate_memory_rejects_malformed_without_gpu():
    import sptrsv_b200 as S

    with pytest.raises(S.SptrsvError) as e:
        S.allocate_memory(np.array([0, 1, 2]), np.array([0, 0]), np.array([1.0, 1.0]), 2)
    assert e.value.code == -3


def test_generators_are_deterministic_and_lower_triangular():
    from sptrsv_b200 import check_csr_host, gen

    for f in (lambda s: gen.banded(3000, 64, 4, 16, seed=s), lambda s: gen.zipf(3000, seed=s),
              lambda s: gen.grid2d(33, 17, seed=s), lambda s: gen.grid3d(7, 5, 6, seed=s),
              lambda s: gen.blockdiag(777, 32, seed=s)):
        a, b, c = f(3), f(3), f(4)
        assert np.array_equal(a.rowptr, b.rowptr) and np.array_equal(a.colidx, b.colidx)
        assert np.array_equal(a.val, b.val)
        assert not (np.array_equal(a.val, c.val) and np.array_equal(a.colidx, c.colidx))
        assert check_csr_host(a.rowptr, a.colidx) == -1


def test_generator_shapes_match_configs():
    from sptrsv_b200 import gen

    g = gen.grid2d(64, 64)
    assert g.n == 4096 and g.nnz == 4096 + 2 * 63 * 64
    d = np.diff(g.rowptr)
    assert d.min() == 1 and d.max() == 3
    assert np.all(g.val[g.rowptr[1:] - 1] == 4.0)
    b = gen.banded(1000, 256, 8, 8, seed=0)
    offs = np.diff(b.rowptr) - 1
    assert np.array_equal(offs, np.minimum(np.arange(1000), 8))
    for i in (300, 999):
        cols = b.colidx[b.rowptr[i]:b.rowptr[i + 1] - 1]
        assert cols.min() >= i - 256 and cols.max() < i
        diag = b.val[b.rowptr[i + 1] - 1]
        assert diag == pytest.approx(1 + np.abs(b.val[b.rowptr[i]:b.rowptr[i + 1] - 1]).sum())
    z = gen.zipf(20000, 1.5, 256, seed=2)
    offs = np.diff(z.rowptr) - 1
    assert offs.max() <= 256 and 0.30 < np.mean(offs == 0) < 0.45  # P(Z=1) = 1/zeta(1.5) = 0.383
    bd = gen.blockdiag(96, 32)
    assert np.array_equal(np.diff(bd.rowptr) - 1, np.tile(np.arange(32), 3))


_NULL_CALLS = """
import ctypes, json
from sptrsv_b200 import _lib as C
L = C.lib()
p = ctypes.c_void_p(0)
calls = [
    ("sptrsv_plan_create", (None, None, ctypes.byref(p))),
    ("sptrsv_plan_set_schedule", (None, None)),
    ("sptrsv_plan_get_schedule", (None, None)),
    ("sptrsv_plan_partition_info", (None, None, None, None, None, None)),
    ("sptrsv_partition_blocks_host", (None, 16, None, None)),
    ("sptrsv_plan_update_values", (None, None)),
    ("sptrsv_solve_f64", (None, None, None, 1, None)),
    ("sptrsv_solve_ir", (None, None, None, 1, None)),
    ("sptrsv_solve_f32", (None, None, None, 1, None)),
    ("sptrsv_plan_calibrate_ir", (None, None, None, 1, 1e-12, 4, None, None)),
    ("sptrsv_solve_host", (None, None, None, 1, 64, None)),
    ("sptrsv_plan_set_stream_segment", (None, 16)),
    ("sptrsv_residual_f64", (None, None, None, None, 1, None)),
    ("sptrsv_solve_ir_noalloc", (None, None, None, 1, None)),
    ("sptrsv_batch_create", (0, None, None, ctypes.byref(p))),
    ("sptrsv_batch_info", (None, None, None, None, None)),
    ("sptrsv_batch_set_schedule", (None, 0, 8, 0, 0, 0)),
    ("sptrsv_batch_set_seq_width", (None, 16.0)),
    ("sptrsv_batch_seq_systems", (None, None, None, None)),
    ("sptrsv_batch_set_partition", (None, 4096)),
    ("sptrsv_batch_partition_info", (None, None, None, None, None)),
    ("sptrsv_batch_solve", (None, None, None, 64, None)),
    ("sptrsv_batch_solve_graph", (None, None, None, 64, None)),
    ("sptrsv_features", (None, None, None)),
    ("sptrsv_schedule_from_class", (-1, None)),
    ("sptrsv_autotune", (None, None, None, 1, 64, 3, None, None)),
    ("sptrsv_mlp_get_params", (None, None)),
    ("sptrsv_mlp_set_params", (None, None)),
    ("sptrsv_mlp_set_normalization", (None, None, None)),
    ("sptrsv_mlp_get_normalization", (None, None, None)),
    ("sptrsv_mlp_forward_host", (None, None, 1, None)),
    ("sptrsv_mlp_gradient_host", (None, None, None, None, 1, None, None)),
    ("sptrsv_mlp_train_host", (None, None, None, None, 1, 1, 1, 1e-3, 0, None)),
    ("sptrsv_mlp_predict_class", (None, None, None)),
    ("sptrsv_plan_select_schedule", (None, None, None, None, None)),
    ("sptrsv_solve_order_tile", (None, None, None, None, 1, None)),
    ("sptrsv_host_spmv", (None, None, None, 1)),
    ("sptrsv_read_mtx_lower", (None, 0, None)),
    ("sptrsv_analysis_levels", (None, None)),
    ("sptrsv_analysis_buckets", (None, None)),
    ("sptrsv_plan_destroy", (None,)),
    ("sptrsv_batch_destroy", (None,)),
    ("sptrsv_mlp_destroy", (None,)),
]
print(json.dumps({name: getattr(L, name)(*args) for name, args in calls}))
"""


def test_null_handles_and_arguments_are_refused_without_a_crash():
    """Every entry point given NULL handles or buffers returns an error code
    (NULL is fine for the destroy functions) instead of dereferencing them;
    the calls run in a child process, so a crash fails this test."""
    import json
    import subprocess
    import sys

    r = subprocess.run([sys.executable, "-c", _NULL_CALLS], cwd=ROOT, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    codes = json.loads(r.stdout.strip().splitlines()[-1])
    for name, code in codes.items():
        if name.endswith("_destroy"):
            assert code == 0, name
        elif name.startswith("sptrsv_analysis_"):
            assert code == -6, (name, code)  # SPTRSV_ERR_NOT_ANALYSED
        else:
            assert code == -2, (name, code)  # SPTRSV_ERR_INVALID_ARG


def test_integration_examples_compile_and_link(tmp_path):
    """The C examples of the integration guide's C section, in order, compile
    as C99 against the header and link against the library (they are not
    run: they need a GPU)."""
    import subprocess

    text = (ROOT / "INTEGRATION.md").read_text()
    text = text[:text.index("## 2.")]  # section 1, the C callers (later sections are other languages' stubs)
    blocks = re.findall(r"```c\n(.*?)```", text, flags=re.S)
    assert len(blocks) >= 5
    body = []
    for blk in blocks:
        # the batch example's nrhs is the per-system array, elsewhere a count
        body.append("{ const int* nrhs = 0;\n" + blk + "}\n" if "sptrsv_batch_create" in blk else blk)
    src = tmp_path / "examples.c"
    src.write_text('#include "sptrsv_b200.h"\n'
                   "int main(void) {\n"
                   "int* rowptr = 0; int* colidx = 0; double* val = 0; int n = 0; double* b = 0; double* x = 0;\n"
                   "double* d_b = 0; double* d_x = 0; int nrhs = 1; cudaStream_t stream = 0;\n"
                   "sptrsv_host_csr_t host_csr = {0}; int nsys = 0; sp_mat_t* mats = 0;\n"
                   + "\n".join(body) + "\nreturn 0;\n}\n")
    exe = tmp_path / "examples"
    lib = ROOT / "sptrsv_b200"
    r = subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", "-Wno-unused-variable", "-Wno-unused-but-set-variable",
                        "-Wno-maybe-uninitialized", "-Wno-uninitialized", f"-I{ROOT / 'include'}", str(src), f"-L{lib}",
                        "-lsptrsv_b200", "-Wl,--allow-shlib-undefined", "-o", str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
