"""bench.py's bookkeeping on the host: the launch count it claims per solve,
the per-configuration summary it attaches to the headline, and the selector
weights' class-table check (no GPU needed)."""
import numpy as np

import bench


class _Sched:
    def __init__(self, variant, partitions):
        self.variant, self.partitions = variant, partitions


def test_solve_launches_count_the_library_kernels():
    # plain: one solve kernel; partitioned: gather, solve, scatter; BAND: b into the records, solve
    assert bench.solve_launches(_Sched(5, 0), 64, 0) == 1
    assert bench.solve_launches(_Sched(5, 16), 64, 0) == 3
    assert bench.solve_launches(_Sched(6, 128), 64, 0) == 2
    assert bench.solve_launches(_Sched(6, 0), 64, 0) == 2
    # FP32 + refinement: a solve per step plus the first, and a residual per step
    assert bench.solve_launches(_Sched(2, 0), 32, 1) == 1 * 2 + 1
    assert bench.solve_launches(_Sched(5, 16), 32, 2) == 3 * 3 + 2


def test_config_summary_keeps_the_figures_of_both_line_kinds():
    single = {"config": {"workload": "w"}, "ms_per_step": 0.5, "value": 2000.0, "dtype": "f64", "steps": 10,
              "schedule": {"name": "band-P128"}, "selected_by": "learned selector (MLP)",
              "rel_err": {"tuned": 1e-15}, "gb_s": 25.0,
              "roofline": {"frac": 0.01, "achieved": 25.0, "traffic": 178495488},
              "e2e": {"value": 1500.0}, "plain_fp64": {"ms": 5.0}, "speedup_vs_plain_fp64": 10.0,
              "clocks": {"reasons": []}, "energy_j_per_solve": 0.1,
              "cpu_baseline": {"value": 2000.0, "cores": 1, "kind": "port"},
              "fp32_refine": {"ms": 0.9}, "fp64_tuned": {"ms": 0.5}}
    out = bench.config_summary(single)
    assert out["ms"] == 0.5 and out["solves_s"] == 2000.0 and out["fp32_refine_ms"] == 0.9
    assert out["fp64_ms"] == 0.5 and out["cpu_ms_per_solve"] == 0.5 and out["e2e_solves_s"] == 1500.0
    assert out["roofline"]["traffic"] == 178495488 and out["roofline"]["frac"] == 0.01
    batch = dict(single, fp32_refine_best_ms=60.0, fp64_best_ms=30.0)
    del batch["fp32_refine"], batch["fp64_tuned"]
    out = bench.config_summary(batch)
    assert out["fp32_refine_ms"] == 60.0 and out["fp64_ms"] == 30.0


def test_selector_weights_of_another_class_table_are_refused(tmp_path, monkeypatch):
    from sptrsv_b200 import select as SEL

    w = tmp_path / "w.npz"
    np.savez(w, params=np.zeros(SEL.N_PARAMS, np.float32), mean=np.zeros(12, np.float32),
             std=np.ones(12, np.float32), table=SEL.CLASS_TABLE - 1)
    monkeypatch.setattr(bench, "SELECTOR_WEIGHTS", w)
    assert not bench.selector_ready(SEL)
    np.savez(w, params=np.zeros(SEL.N_PARAMS, np.float32), mean=np.zeros(12, np.float32),
             std=np.ones(12, np.float32), table=SEL.CLASS_TABLE)
    assert bench.selector_ready(SEL)


def test_traffic_of_every_bench_schedule_is_on_record():
    # the schedules the default run picks: WAVE over 16 blocks (grid), BAND over 128 blocks (banded),
    # the multi-RHS kernel (Zipf, 16 RHS), the batch cut into blocks of 4096 rows
    for key in ("wave_p16_f64_c1", "band_p128_f64_c0", "multirow_f64_c2k16", "batch_p4096_f64_c3"):
        t = bench.load_traffic(key)
        assert isinstance(t, int) and t > 0, key


_REF_ARM = r"""
import json, runpy, sys
sys.argv = ["bench.py", "--impl", "reference", "--config", "c0", "--steps", "2", "--warmup", "3"]
try:
    runpy.run_path("bench.py", run_name="__main__")
except SystemExit as e:
    assert not e.code, e.code
maps = open("/proc/self/maps").read()
print(json.dumps({"mapped": "libsptrsv_b200" in maps, "imported": any(m.startswith("sptrsv_b200") for m in sys.modules)}))
"""


def test_reference_arm_line_and_isolation():
    """The reference arm (CPU, the small banded configuration) prints one line
    with the contract's keys, picks the faster CPU form, and neither imports
    nor maps the product library."""
    import json
    import subprocess
    import sys

    from conftest import ROOT

    r = subprocess.run([sys.executable, "-c", _REF_ARM], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [json.loads(x) for x in r.stdout.strip().splitlines() if x.startswith("{")]
    line, iso = lines[-2], lines[-1]
    assert line["impl"] == "reference" and line["value"] > 0 and line["unit"] == "solves/s"
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["cpu_baseline"]["kind"] == "port"
    assert line["cpu_form"] in ("level", "serial") and line["rel_err_vs_serial"] <= 1e-12
    assert line["probe_ms"][line["cpu_form"]] == min(line["probe_ms"].values())
    assert set(line["config"]) >= {"workload", "n", "nnz", "nlevs", "nrhs"}
    assert iso == {"mapped": False, "imported": False}
