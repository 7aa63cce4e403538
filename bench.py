#!/usr/bin/env python
"""Benchmark: solves/s and HBM GB/s of the B200 SpTRSV on one configuration.

Default workload: the 2D 5-point lower triangle on a 2048x2048 grid
(n = 4,194,304, nnz = 12,578,816, 4095 levels), one right-hand side.

  value         solves/s of the tuned solver (schedule from the learned
                selector when its weights are present, else the exhaustive
                autotuner; precision mode — plain FP64, or FP32 solves with
                FP64 refinement at the calibrated step count — whichever is
                faster), b and x resident in HBM, CUDA events around each
                step, L2 flushed (256 MiB write) before every step.
  fp32_refine   the tuned FP32 + FP64-refinement solve, reported beside it.
  plain_fp64    the drop-in FP64 path (csr_L_solve_multirow) on the same GPU.
  e2e           the tuned solve through the C ABI host-buffer entry point
                (sptrsv_solve_host): pinned host b in, host x out, both copies
                inside the timed region.
  roofline      the dominant kernel: algorithmic bytes per launch / its
                CUDA-event time, against the measured HBM copy bandwidth.
  cpu_baseline  serial FP64 forward substitution (the CPU oracle) on one host
                core, a bounded sample of the same workload.
  reference_kernels  the reference's own solvers built from its sources for
                sm_100a (oracle/_ref), FP64, same matrix, run in a child
                process with a time limit.

--impl reference times the reference algorithm on the host cores instead:
the reference ships no CPU solver, so this is the CPU oracle's
level-scheduled FP64 substitution on all host threads (kind "port").

N > 1 (torchrun): independent replicas, one per GPU, no collective on the
data path; value = all ranks' solves / the slowest rank's time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

import numpy as np  # noqa: E402

CONFIG_NAMES = {
    "c0": "banded n=100000 (8 off-diagonals in a 256 window), 1 RHS",
    "c1": "2D 5-point lower triangle 2048x2048, n=4194304, 1 RHS",
    "c2": "Zipf(1.5) DAG n=2000000 (<=256 off-diagonals), 1 RHS",
    "c2k16": "Zipf(1.5) DAG n=2000000 (<=256 off-diagonals), 16 RHS",
    "c3": "batch of 512 banded systems, n log-uniform [1e3, 2e5], bandwidth log-uniform [16, 4096], "
          "4-16 off-diagonals per row, 1-32 RHS each, one persistent launch replayed as a CUDA graph",
}
TOL = 1e-12
PART_ROWS = (0, 4096)  # batch autotune: plain, and long systems cut into blocks of about 4096 rows
SELECTOR_WEIGHTS = ROOT / "sptrsv_b200" / "selector_weights.npz"


def algorithmic_bytes(n: int, nnz: int, k: int) -> int:
    """Compulsory FP64 bytes of one solve: int32 rowptr, int32 colidx + f64
    values once, f64 b read and f64 x written (k right-hand sides)."""
    return 4 * (n + 1) + 12 * nnz + 16 * n * k


def f32_launch_bytes(n: int, nnz: int, k: int) -> int:
    """Algorithmic bytes of one FP32 solve launch over a plan layout: ptr,
    rowid, FP32 reciprocal diagonal, int32 col + FP32 value per off-diagonal,
    f64 b read, f32 x written."""
    return 4 * (n + 1) + 4 * n + 4 * n + 8 * (nnz - n) + 8 * n * k + 4 * n * k


def solve_launches(sched, mode: int, ir_iters: int) -> int:
    """Kernels of the library launched per solve: the solve kernel, plus a
    gather of b into the block system and a scatter of x out of it when
    partitioned (BAND writes x itself), plus b into BAND's records; FP32 +
    refinement adds a residual and another solve per step."""
    band = sched.variant == 6
    part = sched.partitions >= 2
    one = 2 if band else (3 if part else 1)
    return one if mode == 64 else one * (1 + ir_iters) + ir_iters


def selector_ready(SEL) -> bool:
    """Trained weights for the library's current class table are present."""
    if not SELECTOR_WEIGHTS.exists():
        return False
    z = np.load(SELECTOR_WEIGHTS)
    return (int(z["table"]) if "table" in z.files else 1) == SEL.CLASS_TABLE


def measured_peak():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock / throttle-reason samples during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "50",
                 "-i", str(self.gpu)], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None
        time.sleep(0.3)

    def stop(self):
        if not self.proc:
            return None
        time.sleep(0.1)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = [ln.split(",") for ln in Path(self.path).read_text().splitlines() if ln.strip()]
        os.unlink(self.path)
        sm, smax, reasons, pw = [], 0.0, set(), []
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                smax = max(smax, float(r[2]))
                try:
                    pw.append(float(r[3]))
                except ValueError:
                    pass
                for nm, v in zip(names, r[5:9]):
                    if v.strip().lower() == "active":
                        reasons.add(nm)
            except (ValueError, IndexError):
                continue
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm), "power_w_mean": statistics.mean(pw) if pw else None}


class EnergyMeter:
    """Energy per solve from the GPU's cumulative energy counter (NVML
    nvmlDeviceGetTotalEnergyConsumption, millijoules; a read-only query),
    read before and after a loop of back-to-back solves of at least
    `min_s` seconds: energy delta / solves in that window.  The reference
    samples power in a thread and prints watts per solver
    (source/nvmlPower.cpp:22-59, header/common.h:121); the counter gives the
    energy of exactly the measured window."""

    def __init__(self, torch_mod, device: int):
        self.h = None
        self.note = None
        try:
            import pynvml

            pynvml.nvmlInit()
            pr = torch_mod.cuda.get_device_properties(device)
            bus = f"{pr.pci_domain_id:08X}:{pr.pci_bus_id:02X}:{pr.pci_device_id:02X}.0"
            try:
                self.h = pynvml.nvmlDeviceGetHandleByPciBusId(bus.encode())
            except pynvml.NVMLError:
                self.h = pynvml.nvmlDeviceGetHandleByIndex(device)
            self.nvml = pynvml
        except Exception as e:  # no NVML on this host: report why, measure nothing
            self.note = f"NVML unavailable: {str(e)[:120]}"

    def measure(self, torch_mod, fn, solves_per_call: int, min_s: float = 1.0, stream=None):
        if self.h is None:
            return {"note": self.note}
        fn()
        torch_mod.cuda.synchronize()
        calls = 0
        e0 = self.nvml.nvmlDeviceGetTotalEnergyConsumption(self.h)
        t0 = time.perf_counter()
        while True:
            for _ in range(8):
                fn()
            calls += 8
            torch_mod.cuda.synchronize()
            if time.perf_counter() - t0 >= min_s:
                break
        t1 = time.perf_counter()
        e1 = self.nvml.nvmlDeviceGetTotalEnergyConsumption(self.h)
        joules = (e1 - e0) / 1e3
        solves = calls * solves_per_call
        return {"j_per_solve": joules / solves, "window_s": t1 - t0, "solves": solves,
                "mean_power_w": joules / (t1 - t0),
                "how": "NVML total-energy counter before/after back-to-back solves (no L2 flush)"}


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as td

        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        td.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
        dist = td
    return rank, world, local, dist


def reduce_max(dist, v: float) -> float:
    if dist is None:
        return v
    import torch

    dev = "cuda" if torch.cuda.is_available() and dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([v], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(dist):
    if dist is not None:
        dist.barrier()


# ---------------------------------------------------------------- reference arm
L2_NOTE = "flushed before every step (256 MiB write)"


def workload_config(name: str, n: int, nnz: int, nlevs: int, k: int, world: int) -> dict:
    """The `config` object of a single-system line; both arms print the same one."""
    return {"workload": CONFIG_NAMES[name], "n": n, "nnz": nnz, "nlevs": nlevs, "nrhs": k, "l2": L2_NOTE,
            "parallelism": f"replicas x{world}"}


def batch_workload_config(mats, ks, world: int) -> dict:
    return {"workload": CONFIG_NAMES["c3"], "systems": len(mats), "n_total": int(sum(m.n for m in mats)),
            "nnz_total": int(sum(m.nnz for m in mats)), "rhs_total": int(sum(ks)), "l2": L2_NOTE,
            "parallelism": f"replicas x{world}"}


def host_flush(buf):
    """Evicts the host caches between CPU steps (a 256 MiB write)."""
    buf.fill(1)


def run_reference(args, rank, world, dist):
    """The reference's algorithm on the host cores (CPU oracle): the faster of
    its level-scheduled form on all threads and its serial form on one core.
    Inputs come from the oracle's own copy of the generators, so this arm
    neither imports nor loads the product library."""
    if rank != 0:
        barrier(dist)
        return
    from oracle import oracle as O
    from oracle import workloads as W

    if args.config == "c3":
        run_reference_batch(args, world, dist)
        return
    m, xt, k = W.config(args.config)
    b = m.matvec(xt, k)
    a = O.analysis(m.rowptr, m.colidx)
    lev_ptr = np.concatenate([[0], np.cumsum(np.bincount(a["levels"] - 1, minlength=a["nlevs"]))]).astype(np.int32)
    threads = O.num_threads()
    # two CPU forms of the reference's substitution: level-scheduled on every host thread (a barrier per
    # level) and serial on one core; the arm times the faster of the two on this workload
    forms = {
        "level": (lambda: O.solve_levels_omp(m.rowptr, m.colidx, m.val, b, a["iorder"], lev_ptr, a["nlevs"], k),
                  threads, f"level-scheduled on {threads} threads, {a['nlevs']} levels"),
        "serial": (lambda: O.solve(m.rowptr, m.colidx, m.val, b, nrhs=k), 1, "serial substitution on one core"),
    }
    probe_ms = {}
    for name, (fn, _, _) in forms.items():
        fn()
        t0 = time.perf_counter()
        fn()
        probe_ms[name] = 1e3 * (time.perf_counter() - t0)
    pick = min(probe_ms, key=probe_ms.get)
    solve_fn, threads, how = forms[pick]
    x = solve_fn()
    err = O.rel_err(x, O.solve(m.rowptr, m.colidx, m.val, b, nrhs=k))
    flush_buf = np.empty(256 << 20, dtype=np.uint8)
    for _ in range(args.warmup):
        solve_fn()
    times = []
    for _ in range(args.steps):
        host_flush(flush_buf)
        t0 = time.perf_counter()
        solve_fn()
        times.append(time.perf_counter() - t0)
    total = sum(times)
    v = k * args.steps / total
    sample = (f"{args.steps} full solves of {args.config} ({how}; the faster CPU form in a probe: "
              + ", ".join(f"{f} {t:.2f} ms" for f, t in probe_ms.items()) + ")")
    line = {
        "impl": "reference", "metric": "solves/s", "value": v, "unit": "solves/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload_config(args.config, m.n, m.nnz, a["nlevs"], k, world),
        "cpu_baseline": {"value": v, "unit": "solves/s", "cores": threads, "kind": "port", "sample": sample},
        "e2e": {"value": v, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "gb_s": algorithmic_bytes(m.n, m.nnz, k) * v / 1e9, "rel_err_vs_serial": err, "cpu_form": pick,
        "probe_ms": probe_ms,
    }
    print(json.dumps(line), flush=True)
    barrier(dist)


def run_reference_batch(args, world, dist):
    """Batched configuration on the host cores: the systems are independent,
    so every host thread takes whole systems, each by the serial FP64
    substitution; a step is a bounded sample (the systems in order, a few per
    thread at a time, until about 2 s), value = RHS solved / s."""
    from concurrent.futures import ThreadPoolExecutor

    from oracle import oracle as O
    from oracle import workloads as W

    mats, ks, xs = W.batch_config(512, seed=3)
    threads = O.num_threads()
    prep = [(m, m.matvec(x, k), k) for m, x, k in zip(mats, xs, ks)]
    flush_buf = np.empty(256 << 20, dtype=np.uint8)
    pool = ThreadPoolExecutor(max_workers=threads)  # the oracle's C calls release the GIL

    def solve_one(item):
        m, b, k = item
        O.solve(m.rowptr, m.colidx, m.val, b, nrhs=k)
        return k

    def step():
        host_flush(flush_buf)
        done, t0, i = 0, time.perf_counter(), 0
        while i < len(prep) and time.perf_counter() - t0 < 2.0:
            chunk = prep[i:i + 4 * threads]
            done += sum(pool.map(solve_one, chunk))
            i += len(chunk)
        return done, time.perf_counter() - t0

    for _ in range(args.warmup):
        step()
    done, total = 0, 0.0
    for _ in range(args.steps):
        d, t = step()
        done += d
        total += t
    pool.shutdown()
    v = done / total
    sample = (f"{args.steps} steps, each the systems of the batch in order until 2 s, {threads} threads taking "
              "whole systems (serial substitution each)")
    line = {
        "impl": "reference", "metric": "solves/s", "value": v, "unit": "solves/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": batch_workload_config(mats, ks, world),
        "cpu_baseline": {"value": v, "unit": "solves/s", "cores": threads, "kind": "port", "sample": sample},
        "e2e": {"value": v, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    barrier(dist)


# ---------------------------------------------------------------------- our arm
def event_time_steps(torch, fn, steps, warmup, flush=None, stream=None):
    """Per-step CUDA-event times (ms); the L2 flush runs between steps, outside the events."""
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    evs = []
    for _ in range(steps):
        if flush is not None:
            flush()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        fn()
        e1.record(stream)
        evs.append((e0, e1))
    torch.cuda.synchronize()
    return [a.elapsed_time(b) for a, b in evs]


def cpu_baseline_sample(m, b, k, budget_s=10.0):
    from oracle import oracle as O

    reps, t_total = 0, 0.0
    while reps < 2 or (t_total < budget_s and reps < 200):
        _, dt = O.timed(O.solve, m.rowptr, m.colidx, m.val, b, k)
        reps += 1
        t_total += dt
    return {"value": k * reps / t_total, "unit": "solves/s", "cores": 1, "kind": "port",
            "sample": f"{reps} serial FP64 forward substitutions of the full workload ({t_total:.1f} s)"}


def reference_kernels(cfg: str, timeout_s: int = 240):
    """The reference's solvers (oracle/_ref, built from its sources) on the same
    matrix, in a child process so that a stuck reference kernel cannot take the
    benchmark down; returns {solver: {"ms": median, "err": rel err}} or None."""
    from oracle import oracle as O

    code = (
        "import sys, json; sys.path.insert(0, %r)\n"
        "from oracle import oracle as O\nfrom oracle import workloads as W\n"
        "m, xt, k = W.config(%r)\nb = m.matvec(xt, k)\nref = O.solve(m.rowptr, m.colidx, m.val, b)\nout = {}\n"
        "try:\n"
        "    x, ms, am = O.cusparse_solve(m.rowptr, m.colidx, m.val, b, reps=5)\n"
        "    out['cusparse_spsv'] = {'ms': ms, 'analysis_ms': am, 'rel_err': O.rel_err(x, ref)}\n"
        "except Exception as e:\n"
        "    out['cusparse_spsv'] = {'note': str(e)[:200]}\n"
        "print(json.dumps(out), flush=True)\n"
        "if O.ref_available():\n"
        "    O.ref_lib().ref_set_watchdog_seconds(60.0)\n"
        "    for v, name in ((2, 'ref_multirow'), (1, 'ref_order'), (0, 'ref_simple')):\n"
        "        x, ms = O.ref_solve(v, m.rowptr, m.colidx, m.val, b, reps=5)\n"
        "        out[name] = {'ms': ms, 'rel_err': O.rel_err(x, ref)}\n"
        "        print(json.dumps(out), flush=True)\n" % (str(ROOT), cfg))
    try:
        r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=timeout_s)
    except subprocess.TimeoutExpired as e:
        out = (e.stdout or b"").decode() if isinstance(e.stdout, bytes) else (e.stdout or "")
        lines = [ln for ln in out.splitlines() if ln.startswith("{")]
        return dict(json.loads(lines[-1]), note="timed out") if lines else {"note": "timed out"}
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    if not lines:
        return {"note": f"failed rc={r.returncode}: {r.stderr.strip()[-200:]}"}
    return json.loads(lines[-1])


def chain_hop_us(torch, S, SEL, n=100_000):
    """Per-dependency latency on a bidiagonal chain (one row per level): the
    L2 hop (level-ordered warps, dependency in another SM's row) and the
    shared-memory hop (cluster schedule, dependency in the same CTA)."""
    from sptrsv_b200 import gen

    rp = np.concatenate([[0, 1], 1 + 2 * np.arange(1, n)])
    ci = np.concatenate([[0]] + [[i - 1, i] for i in range(1, n)])
    va = np.ones(ci.shape[0])
    va[rp[1:] - 1] = 2.0
    m = gen.from_arrays(rp, ci, va)
    L = S.allocate_memory(m.rowptr, m.colidx, m.val, n)
    info = S.AnalysisInfo()
    info.mode = S.ALL
    S.run_analysis(info, L)
    plan = S.Plan(L, info)
    b = torch.ones(n, dtype=torch.float64, device="cuda")
    x = torch.empty_like(b)
    out = {}
    for name, sc in (("l2_hop_us", dict(variant=S._lib.VAR_MULTIROW, warps_per_sm=8)),
                     ("smem_hop_us", dict(variant=S._lib.VAR_CLUSTER, rows_per_warp=32, band_levels=4096,
                                          cluster_rows=4096, block_warps=8))):
        plan.set_schedule(**sc)
        t = statistics.median(event_time_steps(torch, lambda: plan.solve_f64(b, x), 3, 1))
        out[name] = 1e3 * t / n
    S.sync_status()
    plan.close()
    S.free_device_analysis(L, info)
    return out


def load_traffic(kernel_key: str):
    p = ROOT / "profiles" / "ncu_traffic.json"
    if p.exists():
        d = json.loads(p.read_text())
        v = d.get(kernel_key)
        if isinstance(v, dict):
            return v.get("dram_bytes_per_launch")
    return None


def run_ours(args, rank, world, local, dist):
    import torch

    import sptrsv_b200 as S
    from oracle import oracle as O
    from sptrsv_b200 import gen
    from sptrsv_b200 import select as SEL

    torch.cuda.set_device(local)
    stream = torch.cuda.current_stream()
    m, xt, k = gen.config(args.config, args.scale if args.lean else 1.0)
    b = m.matvec(xt, k)
    n, nnz = m.n, m.nnz

    L = S.allocate_memory(m.rowptr, m.colidx, m.val, n)
    info = S.AnalysisInfo()
    info.mode = S.ALL
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    S.run_analysis(info, L)
    analysis_ms = 1e3 * (time.perf_counter() - t0)
    plan = S.Plan(L, info)

    db = torch.from_numpy(b).cuda()
    dx = torch.empty(n * k, dtype=torch.float64, device="cuda")
    dx32 = torch.empty(n * k, dtype=torch.float32, device="cuda")
    flush_buf = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")

    def flush():
        flush_buf.fill_(1)

    if args.lean:
        # profiling run: one fixed schedule, warm-up and the timed steps, nothing else
        cls = args.fixed_class if args.fixed_class >= 0 else 4  # wave/G4 over 16 blocks
        s = SEL.schedule_from_class(cls)
        s.ir_max_iters = 1
        plan.set_schedule_struct(s)
        fn = (lambda: plan.solve_f64(db, dx, k)) if args.lean == 64 else (lambda: plan.solve_ir(db, dx, k))
        ts = event_time_steps(torch, fn, args.steps, args.warmup, flush, stream)
        S.sync_status()
        print(json.dumps({"lean": True, "class": SEL.class_name(cls), "precision": args.lean,
                          "ms_per_step": sum(ts) / len(ts)}), flush=True)
        plan.close()
        S.free_device_analysis(L, info)
        return

    # --- schedule: learned selector when trained, exhaustive autotuner beside it
    t0 = time.perf_counter()
    cls64, times64 = SEL.autotune(plan, db, dx, k, 64, reps=3)
    cls32, times32 = SEL.autotune(plan, db, dx, k, 32, reps=3)
    tune_s = time.perf_counter() - t0
    learned = None
    if args.fixed_class >= 0:
        cls64 = cls32 = args.fixed_class
    elif selector_ready(SEL):
        net = SEL.Mlp.load(SELECTOR_WEIGHTS)
        c = net.select(plan, L, info)  # best predicted class that applies to this matrix
        learned = {"class": c, "name": SEL.class_name(c), "time_over_best_fp64": float(times64[c] / times64[cls64])}
        net.close()
    sel64 = learned["class"] if learned else cls64
    sel32 = learned["class"] if learned else cls32
    plan.set_schedule_struct(SEL.schedule_from_class(sel32))
    ir_iters, ir_est = plan.calibrate_ir(db, dx, k, tol=1e-13, max_iters=4)

    def set_mode(mode):
        s = SEL.schedule_from_class(sel64 if mode == 64 else sel32)
        s.ir_max_iters = ir_iters
        plan.set_schedule_struct(s)

    def solve(mode):
        return (lambda: plan.solve_f64(db, dx, k)) if mode == 64 else (lambda: plan.solve_ir(db, dx, k))

    # pick the precision mode by a short measurement
    mode_ms = {}
    for mode in (64, 32):
        set_mode(mode)
        mode_ms[mode] = statistics.median(event_time_steps(torch, solve(mode), 5, 1, flush, stream))
    mode = 64 if mode_ms[64] <= mode_ms[32] else 32
    ref = O.solve(m.rowptr, m.colidx, m.val, b, nrhs=k)
    errs = {}
    for md in (64, 32):
        set_mode(md)
        solve(md)()
        S.sync_status()
        errs[md] = O.rel_err(dx.cpu().numpy(), ref)
    set_mode(mode)

    # --- timed: the tuned solve, device-resident
    sampler = ClockSampler(local)
    barrier(dist)
    torch.cuda.synchronize()
    sampler.start()
    ts = event_time_steps(torch, solve(mode), args.steps, args.warmup, flush, stream)
    clocks = sampler.stop()
    torch.cuda.synchronize()
    barrier(dist)
    S.sync_status()
    total_ms = reduce_max(dist, sum(ts))
    value = world * k * args.steps / (total_ms / 1e3)
    ms_per_step = total_ms / args.steps
    launches_per_step = solve_launches(SEL.schedule_from_class(sel64 if mode == 64 else sel32), mode, ir_iters)

    # --- the other mode and the drop-in FP64 path
    other = 32 if mode == 64 else 64
    set_mode(other)
    t_other = statistics.median(event_time_steps(torch, solve(other), max(5, args.steps // 2), 2, flush, stream))
    set_mode(mode)
    if k == 1:
        fn_plain = lambda: S.csr_L_solve_multirow(L, info, db, dx, n, stream)  # noqa: E731
    else:
        fn_plain = lambda: plan.solve_f64(db, dx, k)  # noqa: E731
    t_plain = statistics.median(event_time_steps(torch, fn_plain, max(5, args.steps // 2), 2, flush, stream))
    S.sync_status()
    err_plain = O.rel_err(dx.cpu().numpy(), ref)
    set_mode(mode)

    # --- dominant kernel and its roofline
    peak, peak_kind = measured_peak()
    if mode == 64:
        t_kern, bytes_kern = ms_per_step, algorithmic_bytes(n, nnz, k)
        kname = "sync-free FP64 solve, one launch per solve (sptrsv_solve_f64)"
    else:
        t_kern = statistics.median(event_time_steps(torch, lambda: plan.solve_f32(db, dx32, k),
                                                    max(5, args.steps // 2), 2, flush, stream))
        bytes_kern = f32_launch_bytes(n, nnz, k)
        kname = "sync-free FP32 solve (sptrsv_solve_f32), 1 + ir_iters launches per solve"
    achieved = bytes_kern / (t_kern / 1e3) / 1e9
    sched = SEL.schedule_from_class(sel64 if mode == 64 else sel32)
    variant = SEL.VARIANT_NAMES[sched.variant]
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": load_traffic(f"{variant}{f'_p{sched.partitions}' if sched.partitions >= 2 else ''}"
                                        f"_{'f64' if mode == 64 else 'f32'}_{args.config}"),
                "kernel": kname, "algorithmic_bytes_per_launch": bytes_kern, "launch_ms": t_kern,
                "peak_kind": peak_kind}
    if not args.extra:
        hops = chain_hop_us(torch, S, SEL)
        roofline.update(hops)
        roofline["latency_floor_ms"] = {"nlevs_x_smem_hop": info.nlevs * hops["smem_hop_us"] / 1e3,
                                        "nlevs_x_l2_hop": info.nlevs * hops["l2_hop_us"] / 1e3}

    # --- end to end through the C ABI host-buffer entry point
    hb = torch.from_numpy(b).pin_memory()
    hx = torch.empty(n * k, dtype=torch.float64).pin_memory()
    te = event_time_steps(torch, lambda: plan.solve_host(hb, hx, k, mode, stream), max(5, args.steps // 2), 2,
                          flush, stream)
    e2e_ms = reduce_max(dist, sum(te)) / len(te)
    err_e2e = O.rel_err(hx.numpy(), ref)

    gbs = algorithmic_bytes(n, nnz, k) / (ms_per_step / 1e3) / 1e9
    energy = EnergyMeter(torch, local).measure(torch, solve(mode), k, min_s=0.5 if args.extra else 1.0)
    cpu = (cpu_baseline_sample(m, b, k, budget_s=4.0 if args.extra else 10.0)
           if (rank == 0 and world == 1 and not args.no_cpu) else None)
    refk = (reference_kernels(args.config)
            if (rank == 0 and world == 1 and not args.no_ref and not args.extra and k == 1) else None)
    t32 = mode_ms[32] if mode == 64 else ms_per_step
    line = {
        "metric": "solves/s", "value": value, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64" if mode == 64 else "f32+f64-refine", "data": "synthetic",
        "config": workload_config(args.config, n, nnz, info.nlevs, k, world),
        "schedule": dict(SEL.schedule_from_class(sel64 if mode == 64 else sel32).as_dict(),
                         ir_max_iters=ir_iters, name=SEL.class_name(sel64 if mode == 64 else sel32)),
        "selected_by": "learned selector (MLP)" if learned else "exhaustive autotuner",
        "gb_s": gbs, "hbm_frac": gbs / peak,
        "rel_err": {"tuned": errs[mode], "fp64": errs[64], "fp32_refine": errs[32], "plain_fp64": err_plain,
                    "e2e": err_e2e, "tol": TOL},
        "fp32_refine": {"solves_s": k / ((t_other if mode == 64 else ms_per_step) / 1e3),
                        "ms": t_other if mode == 64 else ms_per_step, "ir_iters": ir_iters,
                        "calibration_ratio": ir_est},
        "fp64_tuned": {"solves_s": k / ((ms_per_step if mode == 64 else t_other) / 1e3),
                       "ms": ms_per_step if mode == 64 else t_other},
        "plain_fp64": {"solves_s": k / (t_plain / 1e3), "ms": t_plain,
                       "gb_s": algorithmic_bytes(n, nnz, k) / (t_plain / 1e3) / 1e9,
                       "path": "csr_L_solve_multirow" if k == 1 else "sptrsv_solve_f64 (multirow)"},
        "speedup_vs_plain_fp64": t_plain / ms_per_step,
        "fp32_refine_speedup_vs_plain_fp64": t_plain / t32,
        "autotune": {"best_fp64": {"class": cls64, "name": SEL.class_name(cls64), "ms": float(times64[cls64])},
                     "best_fp32_refine": {"class": cls32, "name": SEL.class_name(cls32), "ms": float(times32[cls32])},
                     "seconds": tune_s},
        "learned_selection": learned,
        "analysis_ms": analysis_ms,
        "e2e": {"value": world * k / (e2e_ms / 1e3), "unit": "solves/s", "h2d_bytes_per_step": 8 * n * k,
                "d2h_bytes_per_step": 8 * n * k},
        "energy_j_per_solve": energy.get("j_per_solve"), "energy": energy,
        "roofline": roofline, "gpu_launches": launches_per_step * args.steps,
        "clocks": clocks, "cpu_baseline": cpu, "reference_kernels": refk,
    }
    plan.close()
    S.free_device_analysis(L, info)
    barrier(dist)
    return line


# ------------------------------------------------------------ batched workload
def batch_bytes(mats, ks) -> int:
    return sum(algorithmic_bytes(m.n, m.nnz, k) for m, k in zip(mats, ks))


def batch_e2e_pipelined(torch, batch, prec, db, dx, hb, hx, steps):
    """Milliseconds per step of `steps` batched solves with b copied in from
    pinned host memory and x copied out to it, consecutive steps overlapped:
    copies in on one stream, copies out on another, the solve (a staging
    copy into the graph's b, the graph, a copy of x to staging) on a third.
    Returns (ms per step, 0.0); the caller checks hx."""
    s_in, s_out, stream = torch.cuda.Stream(), torch.cuda.Stream(), torch.cuda.Stream()
    sb = [torch.empty_like(db) for _ in range(2)]
    sx = [torch.empty_like(dx) for _ in range(2)]
    ev_in = [torch.cuda.Event() for _ in range(2)]
    ev_solved = [torch.cuda.Event() for _ in range(2)]
    ev_out = [torch.cuda.Event() for _ in range(2)]
    batch.solve_graph(db, dx, prec)  # the graph for (db, dx) exists before the timed region
    torch.cuda.synchronize()
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0.record(s_in)
    for i in range(steps):
        j = i & 1
        with torch.cuda.stream(s_in):
            if i >= 2:
                s_in.wait_event(ev_solved[j])  # staging b j was taken by step i - 2's solve
            sb[j].copy_(hb, non_blocking=True)
            ev_in[j].record(s_in)
        with torch.cuda.stream(stream):
            stream.wait_event(ev_in[j])
            if i >= 2:
                stream.wait_event(ev_out[j])  # staging x j was read out by step i - 2
            db.copy_(sb[j], non_blocking=True)
            batch.solve_graph(db, dx, prec, stream)
            sx[j].copy_(dx, non_blocking=True)
            ev_solved[j].record(stream)
        with torch.cuda.stream(s_out):
            s_out.wait_event(ev_solved[j])
            hx.copy_(sx[j], non_blocking=True)
            ev_out[j].record(s_out)
    t1.record(s_out)
    torch.cuda.synchronize()
    return t0.elapsed_time(t1) / steps, 0.0


def run_batch(args, rank, world, local, dist):
    """The batched configuration: every system solved in one persistent launch
    per solve (a CUDA graph replay); a step solves all 512 systems with all
    their right-hand sides, so value = sum of right-hand sides / step time."""
    import torch

    import sptrsv_b200 as S
    from oracle import oracle as O
    from sptrsv_b200 import gen
    from sptrsv_b200.batch import Batch

    torch.cuda.set_device(local)
    stream = torch.cuda.current_stream()
    mats, ks, xs = gen.batch_config(args.systems if args.lean else 512, seed=3)
    bs = [m.matvec(x, k) for m, x, k in zip(mats, xs, ks)]
    dev = [S.allocate_memory(m.rowptr, m.colidx, m.val, m.n) for m in mats]
    t0 = time.perf_counter()
    batch = Batch(dev, ks)
    create_s = time.perf_counter() - t0
    nk = sum(ks)
    db = torch.from_numpy(np.concatenate(bs)).cuda()
    dx = torch.empty_like(db)
    flush_buf = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")

    def flush():
        flush_buf.fill_(1)

    if args.lean:
        # profiling run: one schedule (--batch-mode/--batch-width/--batch-bw), warm-up and the timed solves
        prec = args.lean
        batch.set_partition(args.part)
        batch.set_seq_width(args.batch_width)
        batch.set_schedule(mode=args.batch_mode, block_warps=args.batch_bw, ir_iters=1 if prec == 32 else 0)
        ts = event_time_steps(torch, lambda: batch.solve_graph(db, dx, prec), args.steps, args.warmup, flush, stream)
        S.sync_status()
        print(json.dumps({"lean": True, "systems": len(mats), "precision": prec, "ms_per_step": sum(ts) / len(ts)}),
              flush=True)
        return

    refs = [O.solve(m.rowptr, m.colidx, m.val, b, nrhs=k) for m, b, k in zip(mats, bs, ks)]

    def max_err(xh):
        return max(O.rel_err(xh[batch.offsets[s]:batch.offsets[s + 1]], refs[s]) for s in range(len(mats)))

    # --- schedule: level-ordered vs hybrid, block size, refinement steps (exhaustive, small)
    # partitioned (long systems cut into blocks with warm-ups) and plain batches
    cands = []
    for part in PART_ROWS:
        for mode, width in ((0, 0.0), (2, 16.0), (2, 32.0)):
            for bw in (2, 4, 8):
                cands.append((part, mode, width, bw))
    res = {}
    part_info = {}
    for part, mode, width, bw in cands:
        batch.set_partition(part)
        if part not in part_info:
            part_info[part] = batch.partition_info()
        batch.set_seq_width(width)
        for prec, iters in ((64, 0), (32, 1), (32, 2)):
            batch.set_schedule(mode=mode, block_warps=bw, ir_iters=iters)
            t = statistics.median(event_time_steps(torch, lambda: batch.solve_graph(db, dx, prec), 3, 1, flush,
                                                   stream))
            S.sync_status()
            res[(part, mode, width, bw, prec, iters)] = (t, max_err(dx.cpu().numpy()))
    ok = {c: v for c, v in res.items() if v[1] <= TOL}
    best = min(ok, key=lambda c: ok[c][0])
    best64 = min((c for c in ok if c[4] == 64), key=lambda c: ok[c][0])
    best32 = min((c for c in ok if c[4] == 32), key=lambda c: ok[c][0], default=None)

    def apply(c):
        part, mode, width, bw, prec, iters = c
        batch.set_partition(part)
        batch.set_seq_width(width)
        batch.set_schedule(mode=mode, block_warps=bw, ir_iters=iters)

    apply(best)
    prec = best[4]
    sampler = ClockSampler(local)
    barrier(dist)
    torch.cuda.synchronize()
    sampler.start()
    ts = event_time_steps(torch, lambda: batch.solve_graph(db, dx, prec), args.steps, args.warmup, flush, stream)
    clocks = sampler.stop()
    torch.cuda.synchronize()
    barrier(dist)
    S.sync_status()
    err = max_err(dx.cpu().numpy())
    total_ms = reduce_max(dist, sum(ts))
    ms_per_step = total_ms / args.steps
    value = world * nk * args.steps / (total_ms / 1e3)
    nseq, nseqw, nlvl = batch.seq_systems()

    # plain FP64: the level-ordered batched launch, no sequential warps, no blocks
    batch.set_partition(0)
    batch.set_seq_width(0.0)
    batch.set_schedule(mode=0, block_warps=8, ir_iters=1)
    t_plain = statistics.median(event_time_steps(torch, lambda: batch.solve(db, dx, 64), max(3, args.steps // 2), 1,
                                                 flush, stream))
    S.sync_status()
    err_plain = max_err(dx.cpu().numpy())
    apply(best)

    # roofline: one FP64 launch moves the compulsory bytes of every system
    peak, peak_kind = measured_peak()
    nbytes = batch_bytes(mats, ks)
    c64 = best64
    apply(c64)
    t64 = statistics.median(event_time_steps(torch, lambda: batch.solve(db, dx, 64), max(3, args.steps // 2), 1, flush,
                                             stream))
    S.sync_status()
    apply(best)
    achieved = nbytes / (t64 / 1e3) / 1e9
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": load_traffic(f"batch{f'_p{c64[0]}' if c64[0] else ''}_f64_c3"),
                "kernel": "k_sptrsv_vk (one FP64 launch per solve)",
                "algorithmic_bytes_per_launch": nbytes, "launch_ms": t64, "peak_kind": peak_kind,
                "union_levels": batch.nlevs}

    # end to end: pinned host b in, host x out, every step's copies inside the timed region
    hb = torch.from_numpy(np.concatenate(bs)).pin_memory()
    hx = torch.empty(batch.vec_len, dtype=torch.float64).pin_memory()

    def e2e():
        db.copy_(hb, non_blocking=True)
        batch.solve_graph(db, dx, prec)
        hx.copy_(dx, non_blocking=True)

    te = event_time_steps(torch, e2e, max(3, args.steps // 2), 1, flush, stream)
    torch.cuda.synchronize()
    e2e_seq_ms = reduce_max(dist, sum(te)) / len(te)
    err_e2e_seq = max_err(hx.numpy())
    # pipelined across steps (the way a stream of batches is served): step i's b goes in on one copy
    # stream while step i-1 is solved and step i-2's x comes back on another, through two staging
    # buffers per vector; the timed region spans the first step's copy in to the last step's copy out
    n_e2e = max(8, args.steps)  # enough steps that the pipeline's fill and drain weigh little
    e2e_ms, err_e2e = batch_e2e_pipelined(torch, batch, prec, db, dx, hb, hx, n_e2e)
    e2e_ms = reduce_max(dist, e2e_ms * n_e2e) / n_e2e
    err_e2e = max(err_e2e, max_err(hx.numpy()))

    energy = EnergyMeter(torch, local).measure(torch, lambda: batch.solve_graph(db, dx, prec), nk,
                                               min_s=0.5 if args.extra else 1.0)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        done, t_cpu, sys_done = 0, 0.0, 0
        budget = 4.0 if args.extra else 10.0
        for m, b, k in zip(mats, bs, ks):
            _, dt = O.timed(O.solve, m.rowptr, m.colidx, m.val, b, k)
            done += k
            t_cpu += dt
            sys_done += 1
            if t_cpu > budget:
                break
        cpu = {"value": done / t_cpu, "unit": "solves/s", "cores": 1, "kind": "port",
               "sample": f"serial FP64 substitution of the first {sys_done} systems ({done} RHS, {t_cpu:.1f} s)"}
    part, mode, width, bw, _, iters = best
    line = {
        "metric": "solves/s", "value": value, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64" if prec == 64 else "f32+f64-refine", "data": "synthetic",
        "config": batch_workload_config(mats, ks, world),
        "schedule": {"mode": ["level", "chunk", "hybrid"][mode], "seq_width": width, "block_warps": bw,
                     "ir_iters": iters, "sequential_systems": nseq, "sequential_warps": nseqw,
                     "level_rows": nlvl, "nlevs_union": batch.nlevs, "partition_block_rows": part,
                     "partition": part_info.get(part)},
        "selected_by": "exhaustive batch autotune",
        "gb_s": nbytes / (ms_per_step / 1e3) / 1e9, "hbm_frac": nbytes / (ms_per_step / 1e3) / 1e9 / peak,
        "rel_err": {"tuned": err, "plain_fp64": err_plain, "e2e": err_e2e, "tol": TOL},
        "autotune_ms": {f"part{c[0]}/{['level', 'chunk', 'hybrid'][c[1]]}/w{c[2]:g}/bw{c[3]}/p{c[4]}/ir{c[5]}": v[0]
                        for c, v in res.items()},
        "fp64_best_ms": res[best64][0],
        "fp32_refine_best_ms": res[best32][0] if best32 else None,
        "plain_fp64": {"solves_s": nk / (t_plain / 1e3), "ms": t_plain, "path": "level-ordered batched launch"},
        "speedup_vs_plain_fp64": t_plain / ms_per_step,
        "batch_create_s": create_s,
        "e2e": {"value": world * nk / (e2e_ms / 1e3), "unit": "solves/s", "h2d_bytes_per_step": 8 * batch.vec_len,
                "d2h_bytes_per_step": 8 * batch.vec_len, "steps": n_e2e,
                "how": "steps pipelined: copy in, solve and copy out of consecutive steps overlap",
                "sequential_steps": {"value": world * nk / (e2e_seq_ms / 1e3), "ms_per_step": e2e_seq_ms,
                                     "rel_err": err_e2e_seq}},
        "energy_j_per_solve": energy.get("j_per_solve"), "energy": energy,
        "roofline": roofline,
        "gpu_launches": args.steps * ((1 if prec == 64 else 1 + 2 * iters) + (2 if part else 0)),
        "clocks": clocks, "cpu_baseline": cpu,
    }
    batch.close()
    for d in dev:
        S.free_device_analysis(d, None)
    barrier(dist)
    return line


EXTRA_CONFIGS = ("c0", "c2k16", "c3")


def config_summary(line: dict) -> dict:
    """The figures of one configuration's line that ride along the headline."""
    rf = line.get("roofline") or {}
    cpu = line.get("cpu_baseline") or {}
    out = {
        "workload": line["config"]["workload"], "config": line["config"], "ms": line["ms_per_step"],
        "solves_s": line["value"], "dtype": line["dtype"], "steps": line["steps"], "schedule": line.get("schedule"),
        "selected_by": line.get("selected_by"), "rel_err": line["rel_err"], "gb_s": line.get("gb_s"),
        "roofline": {k: rf.get(k) for k in ("achieved", "peak", "frac", "unit", "traffic", "kernel", "launch_ms")},
        "e2e_solves_s": line["e2e"]["value"], "plain_fp64": line.get("plain_fp64"),
        "speedup_vs_plain_fp64": line.get("speedup_vs_plain_fp64"), "clocks": line.get("clocks"),
        "energy_j_per_solve": line.get("energy_j_per_solve"),
        "cpu_baseline": cpu or None,
        "cpu_ms_per_solve": 1e3 / cpu["value"] if cpu.get("value") else None,
    }
    if "fp32_refine" in line and isinstance(line["fp32_refine"], dict):
        out["fp32_refine_ms"] = line["fp32_refine"]["ms"]
        out["fp64_ms"] = line["fp64_tuned"]["ms"]
    else:
        out["fp32_refine_ms"] = line.get("fp32_refine_best_ms")
        out["fp64_ms"] = line.get("fp64_best_ms")
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--config", choices=sorted(CONFIG_NAMES), default="c1")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline sample")
    ap.add_argument("--no-ref", action="store_true", help="skip the reference-kernel comparators")
    ap.add_argument("--fixed-class", type=int, default=-1, help="use this schedule class instead of selecting one")
    ap.add_argument("--lean", type=int, default=0, choices=[0, 32, 64],
                    help="profiling run: only the timed solves of --fixed-class at this precision")
    ap.add_argument("--scale", type=float, default=1.0,
                    help="profiling runs (--lean) only: shrink the configuration's n by this factor")
    ap.add_argument("--no-extra", action="store_true",
                    help="c1 only: skip the other configurations measured after the headline")
    ap.add_argument("--part", type=int, default=0,
                    help="profiling runs (--lean) of c3 only: cut long systems into blocks of about this many rows")
    ap.add_argument("--systems", type=int, default=512,
                    help="profiling runs (--lean) of c3 only: the number of systems in the batch")
    ap.add_argument("--batch-mode", type=int, default=2, choices=[0, 1, 2],
                    help="profiling runs (--lean) of c3 only: 0 level order, 1 natural-order chunks, 2 hybrid")
    ap.add_argument("--batch-width", type=float, default=16.0,
                    help="profiling runs (--lean) of c3 only: the hybrid's mean-level-width threshold")
    ap.add_argument("--batch-bw", type=int, default=4,
                    help="profiling runs (--lean) of c3 only: warps per block")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    args.extra = False
    rank, world, local, dist = dist_setup(args)
    try:
        if args.impl == "reference":
            run_reference(args, rank, world, dist)
            return
        line = (run_batch if args.config == "c3" else run_ours)(args, rank, world, local, dist)
        if line is None:  # a profiling run printed its own line
            return
        if args.config == "c1" and world == 1 and not args.no_extra:
            # the other configurations, measured in the same run (fewer steps)
            line["configs"] = {}
            for cfg in EXTRA_CONFIGS:
                ea = argparse.Namespace(**vars(args))
                ea.config, ea.steps, ea.warmup, ea.extra = cfg, min(args.steps, 10), 3, True
                ea.no_ref = True
                try:
                    ex = (run_batch if cfg == "c3" else run_ours)(ea, rank, world, local, dist)
                    line["configs"][cfg] = config_summary(ex)
                except Exception as e:  # report, keep the headline
                    line["configs"][cfg] = {"error": f"{type(e).__name__}: {str(e)[:300]}"}
        if rank == 0:
            print(json.dumps(line), flush=True)
    finally:
        if dist is not None:
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
