#!/usr/bin/env python
"""Benchmark: solves/s and HBM GB/s of the B200 SpTRSV on one configuration.

Default workload: the 2D 5-point lower triangle on a 2048x2048 grid
(n = 4,194,304, nnz = 12,578,816, 4095 levels), one right-hand side.

  value      solves/s of the tuned FP32 + FP64-refinement solve, b and x
             resident in HBM, CUDA events around each step, L2 flushed
             (256 MiB write) before every step.
  e2e        the same solve through the C ABI host-buffer entry point
             (sptrsv_solve_host): pinned host b in, host x out, both copies
             inside the timed region.
  roofline   the dominant kernel (the FP32 sync-free solve launch):
             algorithmic bytes per launch / its CUDA-event time, against the
             measured HBM copy bandwidth.
  cpu_baseline  serial FP64 forward substitution (the CPU oracle) on one
             host core, a bounded sample of the same workload.
  plain_fp64    the drop-in FP64 path (csr_L_solve_multirow) on the same GPU.

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
}


def algorithmic_bytes(n: int, nnz: int, k: int) -> int:
    """Compulsory FP64 bytes of one solve: int32 rowptr, int32 colidx + f64
    values once, f64 b read and f64 x written (k right-hand sides)."""
    return 4 * (n + 1) + 12 * nnz + 16 * n * k


def f32_launch_bytes(n: int, nnz: int, k: int) -> int:
    """Algorithmic bytes of one FP32 sync-free solve launch over the plan
    layout: ptr, rowid, FP32 diagonal, int32 col + FP32 value per
    off-diagonal, f64 b read, f32 x written."""
    nnz_off = nnz - n
    return 4 * (n + 1) + 4 * n + 4 * n + 8 * nnz_off + 8 * n * k + 4 * n * k


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
        sm, smax, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                smax = max(smax, float(r[2]))
                for nm, v in zip(names, r[5:9]):
                    if v.strip().lower() == "active":
                        reasons.add(nm)
            except (ValueError, IndexError):
                continue
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


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
def run_reference(args, rank, world, dist):
    """The reference's algorithm on the host cores (CPU oracle, all threads)."""
    if rank != 0:
        barrier(dist)
        return
    from oracle import oracle as O
    from sptrsv_b200 import gen

    m, xt, k = gen.config(args.config)
    b = m.matvec(xt, k)
    a = O.analysis(m.rowptr, m.colidx)
    lev_ptr = np.concatenate([[0], np.cumsum(np.bincount(a["levels"] - 1, minlength=a["nlevs"]))]).astype(np.int32)
    threads = O.num_threads()
    x = O.solve_levels_omp(m.rowptr, m.colidx, m.val, b, a["iorder"], lev_ptr, a["nlevs"], k)
    err = O.rel_err(x, O.solve(m.rowptr, m.colidx, m.val, b, nrhs=k))
    for _ in range(args.warmup):
        O.solve_levels_omp(m.rowptr, m.colidx, m.val, b, a["iorder"], lev_ptr, a["nlevs"], k)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        O.solve_levels_omp(m.rowptr, m.colidx, m.val, b, a["iorder"], lev_ptr, a["nlevs"], k)
        times.append(time.perf_counter() - t0)
    total = sum(times)
    v = k * args.steps / total
    sample = f"{args.steps} full solves of {args.config} (level-scheduled, {a['nlevs']} levels)"
    line = {
        "impl": "reference", "metric": "solves/s", "value": v, "unit": "solves/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": CONFIG_NAMES[args.config], "n": m.n, "nnz": m.nnz, "nrhs": k},
        "cpu_baseline": {"value": v, "unit": "solves/s", "cores": threads, "kind": "port", "sample": sample},
        "e2e": {"value": v, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "gb_s": algorithmic_bytes(m.n, m.nnz, k) * v / 1e9, "rel_err_vs_serial": err,
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

    torch.cuda.set_device(local)
    stream = torch.cuda.current_stream()
    m, xt, k = gen.config(args.config)
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

    # schedule: short sweep of the FP32 solve over the variants (autotuned pick)
    cands = [(S._lib.VAR_MULTIROW, 1)] + [(v, r) for v in (S._lib.VAR_ORDER, S._lib.VAR_SIMPLE)
                                           for r in (1, 2, 4, 8, 16, 32)]
    best = None
    for var, rpw in cands:
        plan.set_schedule(var, rpw, ir_max_iters=2)
        ts = event_time_steps(torch, lambda: plan.solve_f32(db, dx32, k), 3, 1, flush, stream)
        t = statistics.median(ts)
        if best is None or t < best[0]:
            best = (t, var, rpw)
    plan.set_schedule(best[1], best[2], ir_max_iters=2)
    S.sync_status()

    # correctness of the timed paths against the FP64 oracle
    ref = O.solve(m.rowptr, m.colidx, m.val, b, nrhs=k)
    plan.solve_ir(db, dx, k)
    S.sync_status()
    err_ir = O.rel_err(dx.cpu().numpy(), ref)
    plan.solve_f64(db, dx, k)
    S.sync_status()
    err_f64 = O.rel_err(dx.cpu().numpy(), ref)

    # timed: FP32 + FP64 refinement, device-resident
    sampler = ClockSampler(local) if rank == 0 or world > 1 else None
    barrier(dist)
    torch.cuda.synchronize()
    if sampler:
        sampler.start()
    ts = event_time_steps(torch, lambda: plan.solve_ir(db, dx, k), args.steps, args.warmup, flush, stream)
    clocks = sampler.stop() if sampler else None
    torch.cuda.synchronize()
    barrier(dist)
    S.sync_status()
    total_ms = reduce_max(dist, sum(ts))
    value = world * k * args.steps / (total_ms / 1e3)

    # dominant kernel: the FP32 sync-free solve launch
    t32 = statistics.median(event_time_steps(torch, lambda: plan.solve_f32(db, dx32, k), max(5, args.steps // 2),
                                             2, flush, stream))
    peak, peak_kind = measured_peak()
    b32 = f32_launch_bytes(n, nnz, k)
    achieved = b32 / (t32 / 1e3) / 1e9
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": load_traffic(f"sptrsv_f32_{args.config}"), "kernel": "k_sptrsv<PermMat<float>> (FP32 solve)",
                "algorithmic_bytes_per_launch": b32, "launch_ms": t32, "peak_kind": peak_kind}

    # plain FP64 sync-free solve (the drop-in path)
    if k == 1:
        t64p = event_time_steps(torch, lambda: S.csr_L_solve_multirow(L, info, db, dx, n, stream),
                                max(5, args.steps // 2), 2, flush, stream)
    else:
        t64p = event_time_steps(torch, lambda: plan.solve_f64(db, dx, k), max(5, args.steps // 2), 2, flush, stream)
    S.sync_status()
    plain_ms = statistics.median(t64p)
    plain = {"solves_s": k / (plain_ms / 1e3), "ms": plain_ms,
             "gb_s": algorithmic_bytes(n, nnz, k) / (plain_ms / 1e3) / 1e9,
             "path": "csr_L_solve_multirow" if k == 1 else "sptrsv_solve_f64"}

    # end to end through the C ABI host-buffer entry point
    hb = torch.from_numpy(b).pin_memory()
    hx = torch.empty(n * k, dtype=torch.float64).pin_memory()
    te = event_time_steps(torch, lambda: plan.solve_host(hb, hx, k, 32, stream), max(5, args.steps // 2),
                          2, flush, stream)
    e2e_ms = reduce_max(dist, sum(te)) / len(te)
    err_e2e = O.rel_err(hx.numpy(), ref)

    ms_per_step = total_ms / args.steps
    gbs = algorithmic_bytes(n, nnz, k) / (ms_per_step / 1e3) / 1e9
    cpu = cpu_baseline_sample(m, b, k) if (rank == 0 and world == 1 and not args.no_cpu) else None
    sched_names = {0: "simple", 1: "order", 2: "multirow", 3: "cluster"}
    line = {
        "metric": "solves/s", "value": value, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32+f64-refine", "data": "synthetic",
        "config": {"workload": CONFIG_NAMES[args.config], "n": n, "nnz": nnz, "nlevs": info.nlevs, "nrhs": k,
                   "l2": "flushed before every step (256 MiB write)",
                   "schedule": {"variant": sched_names[best[1]], "rows_per_warp": best[2], "ir_iters": 2},
                   "parallelism": f"replicas x{world}"},
        "gb_s": gbs, "hbm_frac": gbs / peak, "rel_err": {"fp32_ir": err_ir, "fp64": err_f64, "e2e": err_e2e},
        "plain_fp64": plain, "speedup_vs_plain_fp64": plain_ms / ms_per_step,
        "analysis_ms": analysis_ms,
        "e2e": {"value": world * k / (e2e_ms / 1e3), "unit": "solves/s", "h2d_bytes_per_step": 8 * n * k,
                "d2h_bytes_per_step": 8 * n * k},
        "roofline": roofline, "gpu_launches": (1 + 2 * 2) * args.steps,
        "clocks": clocks, "cpu_baseline": cpu,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    plan.close()
    S.free_device_analysis(L, info)
    barrier(dist)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--config", choices=sorted(CONFIG_NAMES), default="c1")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline sample")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    rank, world, local, dist = dist_setup(args)
    try:
        if args.impl == "reference":
            run_reference(args, rank, world, dist)
        else:
            run_ours(args, rank, world, local, dist)
    finally:
        if dist is not None:
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
