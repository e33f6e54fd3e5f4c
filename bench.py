"""Benchmark of the SparseOps hot path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (one "step" = one SpMV y = A*x over the whole matrix): the power-law
configuration -- FP64 CSR, n = 4,194,304 square, row lengths
round(lognormal(ln 12, 1.2)) clipped to [1, 20000], columns uniform without
replacement, values N(0,1), x uniform[-1,1], seed 1 -- seeded synthetic data
(the reference's SuiteSparse inputs are not available).

Metric: achieved HBM GB/s on the ALGORITHMIC bytes of one SpMV,
    4*(n+1) + (4+8)*nnz + 8*n_cols + 8*n_rows
(row offsets, column indices, values, x once, y written), and its fraction of
the measured HBM copy bandwidth (MEASURED_PEAKS.json).  The matrix (about
1.3 GB) is larger than the 126 MB L2, so no flush is needed between steps.

  value     device-resident: matrix, x and y already in HBM; K back-to-back
            SpMVs timed with CUDA events on the launching stream.
  e2e       the C ABI host path (spops_spmv_host): pinned host x uploaded, the
            SpMV, y downloaded, every step.
  cpu_baseline  the reference's own OpenMP CSR kernel (oracle/_ref, compiled
            from the reference sources; kernel_flag 2) on this host's cores,
            on a bounded sample of the same workload (rank 0, N = 1 only).

--impl reference runs only the reference CPU kernel (all host threads).
--gpus N > 1: launched under torchrun, every rank runs an independent replica
(the path does not shard: "replicas only"); value = all ranks' bytes / the
max-over-ranks time.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "SpMV HBM GB/s (% of peak); batched & fwd+bwd speedup vs plain, rel err ≤1e-12"
N_ROWS = 4194304
PEAK_FALLBACK = 6650.0


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return PEAK_FALLBACK, "fallback"


def workload(rows=N_ROWS):
    from sparseops_b200 import synth
    rp, ci, v = synth.powerlaw(rows, mu=math.log(12.0), sigma=1.2, lo=1, hi=20000, seed=1)
    x = synth.uniform(rows, 1)
    return rp, ci, v, x


def spmv_bytes(n_rows, n_cols, nnz, isz=4, vsz=8):
    return isz * (n_rows + 1) + (isz + vsz) * nnz + vsz * n_cols + vsz * n_rows


def profile_traffic(name="csr_tile_kernel_powerlaw.txt"):
    """DRAM bytes per launch from the committed ncu summary, if present."""
    p = os.path.join(ROOT, "profiles", name)
    try:
        for line in open(p):
            if line.startswith("dram_bytes_per_launch"):
                return float(line.split("=")[1].split()[0])
    except OSError:
        pass
    return None


class Clocks:
    """Samples nvidia-smi during the timed region."""

    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, dev):
        self.dev, self.p = dev, None

    def start(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "100"],
                                      stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except (OSError, ValueError):
            self.p = None

    def stop(self):
        if self.p is None:
            return None
        self.p.terminate()
        try:
            out, _ = self.p.communicate(timeout=5)
        except subprocess.TimeoutExpired:
            self.p.kill()
            out, _ = self.p.communicate()
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.strip().splitlines():
            f = [t.strip() for t in line.split(",")]
            if len(f) < 7:
                continue
            try:
                sm.append(float(f[0]))
                mx = max(mx, float(f[1]))
            except ValueError:
                continue
            for nm, val in zip(names, f[3:7]):
                if val.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def max_over_ranks(x: float, dist, device) -> float:
    """Max of a per-rank time over all ranks (identity without a process group)."""
    if dist is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_gbs(world: int, nbytes: int, ms: float) -> float:
    """Replicas: every rank processes `nbytes`; the job takes the slowest rank's time."""
    return world * nbytes / (ms * 1e-3) / 1e9


def cpu_reference_sample(rp, ci, v, x, budget_s=10.0, threads=None):
    """Time the reference's CSR kernel (flag 2) on host cores on a row slab of
    the workload sized to about `budget_s` of CPU work.  Returns (GB/s, info)."""
    from oracle import Reference, reference_available
    if reference_available():
        R = Reference(threads=threads or os.cpu_count())
        kind = "reference"

        def run(rp_, ci_, v_, x_, y_):
            R.spmv_csr(rp_, ci_, v_, x_, 1.0, 0.0, None, flag=2, out=y_)
    else:  # the oracle's sequential restatement
        from oracle import Oracle
        O = Oracle()
        kind = "port"
        threads = 1

        def run(rp_, ci_, v_, x_, y_):
            O.spmv_csr(rp_, ci_, v_, x_)
    n = len(rp) - 1
    # calibrate on 1/64 of the rows
    m = max(1, n // 64)
    t0 = time.perf_counter()
    ybuf = np.zeros(n)
    run(rp[:m + 1], ci[:rp[m]], v[:rp[m]], x, ybuf[:m])
    t1 = max(time.perf_counter() - t0, 1e-4)
    per_full = t1 * (rp[-1] / max(rp[m], 1))
    iters = max(1, min(50, int(budget_s / max(per_full, 1e-6))))
    frac = 1.0 if per_full * iters <= budget_s * 1.5 else budget_s / per_full
    m = n if frac >= 1.0 else max(1, int(n * frac))
    rps, cis, vs = rp[:m + 1], ci[:rp[m]], v[:rp[m]]
    touched = int(np.count_nonzero(np.bincount(cis, minlength=len(x)))) if m < n else len(x)
    nbytes = 4 * (m + 1) + 12 * int(rps[-1]) + 8 * touched + 8 * m
    run(rps, cis, vs, x, ybuf[:m])  # warm-up
    t0 = time.perf_counter()
    for _ in range(iters):
        run(rps, cis, vs, x, ybuf[:m])
    dt = (time.perf_counter() - t0) / iters
    return nbytes / dt / 1e9, dict(kind=kind, cores=int(threads or os.cpu_count()),
                                   sample=f"rows [0,{m}) of {n} ({int(rps[-1])} nnz), {iters} SpMV")


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    t0 = time.time()
    rp, ci, v, x = workload(args.rows)
    log(f"workload built in {time.time() - t0:.1f}s, nnz={len(ci)}")
    from oracle import Reference, reference_available
    if not reference_available():
        print(json.dumps({"impl": "reference", "unavailable": "reference library (oracle/_ref) not built"}))
        return 0
    threads = os.cpu_count()
    R = Reference(threads=threads)
    n = len(rp) - 1
    full = spmv_bytes(n, n, len(ci))
    y = np.zeros(n)
    t0 = time.perf_counter()
    R.spmv_csr(rp, ci, v, x, 1.0, 0.0, y, flag=2)
    t_full = time.perf_counter() - t0
    # each step is a bounded sample: the whole matrix if K steps fit ~2 minutes
    budget = 120.0 / max(1, args.steps + args.warmup)
    if t_full <= budget:
        m, sample = n, "whole matrix per step"
    else:
        m = max(1, int(n * budget / t_full))
        sample = f"rows [0,{m}) of {n} per step"
    rps, cis, vs = rp[:m + 1], ci[:rp[m]], v[:rp[m]]
    touched = int(np.count_nonzero(np.bincount(cis, minlength=n))) if m < n else n
    nbytes = 4 * (m + 1) + 12 * int(rps[-1]) + 8 * touched + 8 * m if m < n else full
    ys = np.zeros(m)
    for _ in range(args.warmup):
        R.spmv_csr(rps, cis, vs, x, 1.0, 0.0, None, flag=2, out=ys)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        R.spmv_csr(rps, cis, vs, x, 1.0, 0.0, None, flag=2, out=ys)
    dt = (time.perf_counter() - t0) / args.steps
    gbs = nbytes / dt / 1e9
    peak, _ = peaks()
    out = {
        "impl": "reference", "metric": METRIC, "value": round(gbs, 2), "unit": "GB/s", "n_gpus": 0,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(dt * 1e3, 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"powerlaw CSR SpMV FP64 n={n} (lognormal ln12,1.2; seed 1)",
                   "nnz": int(len(ci)), "kernel_flag": 2},
        "pct_of_peak": round(100 * gbs / peak, 2),
        "cpu_baseline": {"value": round(gbs, 2), "unit": "GB/s", "cores": threads, "kind": "reference",
                         "sample": sample},
        "e2e": {"value": round(gbs, 2), "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out))
    return 0


def run_ours(args):
    import torch
    import ctypes as C
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    from sparseops_b200 import CSR_Matrix, default_context
    from sparseops_b200._lib import call, dbl, vp

    t0 = time.time()
    rp, ci, v, x = workload(args.rows)
    n, nnz = len(rp) - 1, len(ci)
    log(f"[rank {rank}] workload built in {time.time() - t0:.1f}s: n={n} nnz={nnz}")
    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream(dev)
    ctx = default_context(local)
    if args.csr_variant:
        ctx.set_option("csr_variant", args.csr_variant)
    A = CSR_Matrix(n, n, rp, ci, v)
    h = A.device(ctx)
    xd = torch.from_numpy(x).to(dev)
    yd = torch.zeros(n, dtype=torch.float64, device=dev)
    nbytes = spmv_bytes(n, n, nnz)

    def step():
        call("spops_spmv", ctx.handle, dbl(1.0), h.handle, vp(xd.data_ptr()), dbl(0.0), vp(yd.data_ptr()))

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clocks = Clocks(local)
    clocks.start()
    time.sleep(0.3)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    ev0.record(stream)
    for _ in range(args.steps):
        step()
    ev1.record(stream)
    torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1) / args.steps
    ck = clocks.stop()
    ms = max_over_ranks(ms, dist, dev)
    if dist:
        dist.barrier()
    value = whole_job_gbs(world, nbytes, ms)

    # ---- e2e: the host path through the C ABI (pinned x in, y out, per step)
    xh = torch.from_numpy(x).pin_memory()
    yh = torch.zeros(n, dtype=torch.float64).pin_memory()
    e2e_steps = max(3, min(args.steps, 200))

    def step_host():
        call("spops_spmv_host", ctx.handle, dbl(1.0), h.handle, vp(xh.data_ptr()), dbl(0.0), vp(yh.data_ptr()))

    for _ in range(max(3, args.warmup // 10)):
        step_host()
    if dist:
        dist.barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(e2e_steps):
        step_host()
    e1.record(stream)
    torch.cuda.synchronize()
    ems = max_over_ranks(e0.elapsed_time(e1) / e2e_steps, dist, dev)
    e2e = whole_job_gbs(world, nbytes, ems)
    # correctness spot check of the e2e result against the device result
    ok = bool(torch.equal(yh.to(dev), yd))

    peak, peak_kind = peaks()
    traffic = profile_traffic()
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            gbs, info = cpu_reference_sample(rp, ci, v, x, budget_s=args.cpu_budget)
            cpu = dict(value=round(gbs, 3), unit="GB/s", **info)
        except Exception as e:  # keep the line even if the baseline cannot run
            cpu = {"value": None, "unit": "GB/s", "error": str(e)[:200]}
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return 0
    out = {
        "metric": METRIC, "value": round(value, 2), "unit": "GB/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms, 5), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"powerlaw CSR SpMV FP64 n={n} (lognormal ln12,1.2 clip [1,20000]; seed 1)",
                   "nnz": int(nnz), "algorithmic_bytes_per_step": int(nbytes),
                   "l2": "inputs larger than L2 (matrix ~1.3 GB vs 126 MB), no flush",
                   "parallelism": "replicas" if world > 1 else "single GPU"},
        "pct_of_peak": round(100 * value / world / peak, 2),
        "roofline": {"bound": "hbm", "achieved": round(nbytes / (ms * 1e-3) / 1e9, 2), "peak": peak,
                     "unit": "GB/s", "frac": round(nbytes / (ms * 1e-3) / 1e9 / peak, 4),
                     "peak_source": peak_kind,
                     "kernel": "csr_tile_kernel<int,double,8,3,1> + csr_tile_calibrate_kernel<double>",
                     "traffic": traffic},
        "e2e": {"value": round(e2e, 2), "unit": "GB/s", "h2d_bytes_per_step": 8 * n, "d2h_bytes_per_step": 8 * n,
                "steps": e2e_steps, "matches_device_result": ok,
                "path": "spops_spmv_host (matrix resident after first upload)"},
        # tile kernel + its calibrator per SpMV; one launch for the segment kernel
        "gpu_launches": args.steps * (1 if args.csr_variant in (2, 3, 4) else 2),
        "clocks": ck,
        "cpu_baseline": cpu,
    }
    print(json.dumps(out))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=4000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-budget", type=float, default=10.0)
    ap.add_argument("--csr-variant", type=int, default=0, help="CSR kernel shape (spops_set_option)")
    ap.add_argument("--rows", type=int, default=N_ROWS,
                    help="matrix rows (default: the benchmark size; smaller only for profiling captures)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
