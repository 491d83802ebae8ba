#!/usr/bin/env python3
"""Throughput benchmark of the BEAM bispectrum estimator hot path on B200.

Workload: one bispectrum = all 16 (l,m) multipoles over all (k1, t, mu) bins of
one realization at NN=384, Nmax=100 planes, Nr=40 rings, k1 bins 1..51 of
width 1, 5 t and mu bins: the reference example `barbie 384 1 51 1 1`.
Inputs are seeded synthetic fields in the reference's r2c input layout (no
public dataset is involved).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Our arm prints one JSON line: `value` is bispectra/hour with the r2c buffers
resident in HBM (the plain FP64 path, 1e-10 of the reference); `e2e` is the
same through the C ABI from pinned host buffers (host gather + H2D + compute +
D2H of the bins); `mixed` is the FP32 path with its error against FP64 per
(l,m,bin); `roofline` is the triangle-sum kernel against the measured FP64
peak; `cpu_baseline` is the oracle's CPU restatement timed on a bounded sample.
Each rank processes its own realizations (weak scaling, no collective on the
data path).

The reference arm (--impl reference) times the reference program itself
(oracle/_ref/barbie_ref, built from the reference's sources) on bounded
samples of the same workload on the host cores, rank 0 only.
"""
from __future__ import annotations

import argparse
import json
import os
import re
import shutil
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = dict(NN=384, Nmax=100, Nr=40, UL_k1=51, LL_k1=1, BW_k1=1, n_mtbin=5)
METRIC = "bispectra/hour @NN=384 (mixed vs FP64, 1 B200, rel err<=1e-5); p50/p99 latency"
UNIT = "bispectra/hour"
WORKLOAD_NAME = "barbie 384 1 51 1 1: NN=384, Nmax=100, Nr=40, k1 bins 1..51 width 1, 5 t x 5 mu bins, 16 (l,m)"


def parse_args():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--fields", type=int, default=2, help="realizations per rank, cycled over the steps")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-mixed", action="store_true")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched form (64 realizations at NN=256)")
    ap.add_argument("--no-serve", action="store_true", help="skip the serving form (Poisson job stream)")
    ap.add_argument("--no-field", action="store_true", help="skip the field generation / ingestion timing")
    ap.add_argument("--no-autotune", action="store_true",
                    help="keep the default work decomposition and FFT tiles (no beam_gpu_*_autotune)")
    ap.add_argument("--serve-jobs", type=int, default=200, help="jobs per precision in the serving stream")
    ap.add_argument("--batch-pool", type=int, default=64, help="distinct fields cycled over the batch")
    return ap.parse_args()


# batched form: 64 realizations of the field recipe at NN=256, Nr=30 rings, mixed precision
BATCH = dict(NN=256, Nmax=64, Nr=30, UL_k1=31, LL_k1=1, BW_k1=1, n_mtbin=5, realizations=64)
# serving form: NN -> (Nmax, Nr) with the ring extent Nmax below NN/3 and above the
# last ring's lower edge (27.9, 56.9, 95.9 for Nr = 20, 30, 40); bins 1..Nmax of width 1 or 2
SERVE = {128: (40, 20), 192: (60, 30), 256: (64, 30), 384: (100, 40), 512: (128, 40)}


# --------------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi clock/throttle samples every 200 ms while running."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(prefix="beam_clocks_", suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}", "--format=csv,noheader",
                 "-lms", "200", "-f", self.path], stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.3)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = []
        with open(self.path) as fh:
            for line in fh:
                f = [x.strip() for x in line.split(",")]
                if len(f) >= 9 and f[1].split()[0].isdigit():
                    rows.append(f)
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [int(r[1].split()[0]) for r in rows]
        mx = [int(r[2].split()[0]) for r in rows]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower() == "active"})
        power = [float(r[3].split()[0]) for r in rows if r[3].split()[0].replace(".", "").isdigit()]
        return {"sm_mhz": int(statistics.median(sm)), "sm_max_mhz": max(mx), "reasons": reasons,
                "samples": len(rows), "power_w_max": max(power) if power else None}


# ------------------------------------------------------------------- helpers
def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def measured_fp64_peak(torch, device) -> float:
    """cuBLAS DGEMM throughput (TFLOP/s), best of 5 at 8192^3."""
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device=device)
    b = torch.randn(n, n, dtype=torch.float64, device=device)
    torch.matmul(a, b)
    torch.cuda.synchronize()
    best = float("inf")
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1))
    del a, b
    torch.cuda.empty_cache()
    return 2.0 * n ** 3 / (best / 1e3) / 1e12


def measured_fp32_peak(torch, device) -> float:
    """cuBLAS SGEMM throughput (TFLOP/s) with TF32 off, i.e. FP32 FMA on the
    CUDA cores: best of 5 at 8192^3."""
    n = 8192
    prev = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = False
    try:
        a = torch.randn(n, n, dtype=torch.float32, device=device)
        b = torch.randn(n, n, dtype=torch.float32, device=device)
        torch.matmul(a, b)
        torch.cuda.synchronize()
        best = float("inf")
        for _ in range(5):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            torch.matmul(a, b)
            e1.record()
            torch.cuda.synchronize()
            best = min(best, e0.elapsed_time(e1))
        del a, b
        torch.cuda.empty_cache()
    finally:
        torch.backends.cuda.matmul.allow_tf32 = prev
    return 2.0 * n ** 3 / (best / 1e3) / 1e12


def triangle_flops(info) -> float:
    """Algorithmic flops of one bispectrum's triangle sums: a complex
    multiply-accumulate per closed in-plane triangle term (x_k1 z_k3 into the
    run's outer product: 8 flop), and per (run, accepted triangle) the product
    with the run's third leg, Re(y W), added to the triangle's sum (4 flop)."""
    return 8.0 * info["n_fourier_terms"] + 4.0 * info["n_run_combos"]


def profile_traffic(kernel: str):
    """DRAM bytes per launch of a kernel from a committed ncu summary, if any."""
    path = os.path.join(ROOT, "profiles", f"{kernel}_nn384.md")
    if not os.path.exists(path):
        return None
    with open(path) as fh:
        for line in fh:
            m = re.search(r"dram_bytes_per_launch\s*=\s*([0-9.eE+]+)", line)
            if m:
                return float(m.group(1))
    return None


def mixed_errors(fp64: dict, mixed: dict) -> dict:
    """Relative error of the mixed path against FP64 per (l,m,bin), printed bins only."""
    ok = (fp64["norm"][..., 0] > 0.1)[..., None] & np.isfinite(fp64["out"]) & (fp64["out"] != 0)
    ok = np.broadcast_to(ok, fp64["out"].shape)
    rel = np.full(fp64["out"].shape, np.nan)
    rel[ok] = np.abs(mixed["out"][ok] - fp64["out"][ok]) / np.abs(fp64["out"][ok])
    per_lm = [float(np.nanmax(rel[..., k])) if np.any(ok[..., k]) else None for k in range(16)]
    r = rel[ok]
    return {"max_rel_err": float(r.max()), "p99_rel_err": float(np.quantile(r, 0.99)),
            "median_rel_err": float(np.median(r)), "frac_within_1e-5": float(np.mean(r <= 1e-5)),
            "max_rel_err_per_lm": per_lm, "bins_compared": int(r.size),
            "counts_identical": bool(np.array_equal(fp64["count"], mixed["count"]))}


def oracle_fixture_bins(field):
    """Bins of the committed oracle fixture of the benchmark workload
    (tests/golden/oracle_nn384_cfg3.npz: the oracle's pixel sums on the
    benchmark's first field), shaped as a run's result, or None when the
    fixture is absent or belongs to another field."""
    import hashlib
    path = os.path.join(ROOT, "tests", "golden", "oracle_nn384_cfg3.npz")
    if not os.path.exists(path):
        return None
    g = np.load(path)
    if str(g["field_sha256"]) != hashlib.sha256(field.tobytes()).hexdigest():
        return None
    vol = float(WORKLOAD["NN"]) ** 3
    with np.errstate(divide="ignore", invalid="ignore"):
        out = g["bs"] / (vol * g["norm"])
    return {"out": out, "norm": g["norm"], "count": g["counts"]}


# --------------------------------------------------------------------- ours
def run_ours(args):
    import torch
    import torch.distributed as dist

    from barbie_b200 import beam
    from barbie_b200.synth import realization_seed, synth_field

    world, rank, local = dist_setup(args)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    W = WORKLOAD
    ctx = beam.Context(local)
    fields = [synth_field(W["NN"], realization_seed(1 + rank * args.fields + i)) for i in range(args.fields)]
    dev_fields = [torch.from_numpy(f).to(dev) for f in fields]
    host_fields = [torch.from_numpy(f).pin_memory() for f in fields]
    host_np = [h.numpy() for h in host_fields]
    torch.cuda.synchronize(dev)
    # cold start: plan creation (geometry, triangle lists, work decomposition;
    # no autotuning) and the first bispectrum from a pinned host field, host clock
    t0 = time.perf_counter()
    plan = beam.Plan(ctx, W["NN"], W["UL_k1"], W["LL_k1"], W["BW_k1"], Nmax=W["Nmax"], Nr=W["Nr"],
                     n_mtbin=W["n_mtbin"])
    t1 = time.perf_counter()
    plan.run(host_np[0])
    t2 = time.perf_counter()
    cold = {"plan_create_ms": (t1 - t0) * 1e3, "first_run_ms": (t2 - t1) * 1e3, "total_ms": (t2 - t0) * 1e3,
            "phases_ms": dict(zip(("geometry", "triangle_lists", "work", "tables", "run_buffers"),
                                  plan.info["build_ms"]))}
    tuning = {"fp64": tune_plan(plan, args)}
    info = plan.info
    stream = torch.cuda.ExternalStream(ctx.stream, device=dev)

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize(dev)

    def max_over_ranks(x: float) -> float:
        if world == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)  # 256 MiB > L2

    def timed_loop(p, srcs, steps):
        times, tri = [], []
        for i in range(steps):
            with torch.cuda.stream(stream):
                flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            p.run(srcs[i % len(srcs)])
            e1.record(stream)
            e1.synchronize()
            times.append(e0.elapsed_time(e1))
            tri.append(p.last_timings()["triangle"])
        return times, tri

    # warm-up, then the timed device-resident loop
    timed_loop(plan, dev_fields, args.warmup)
    barrier()
    clocks = ClockSampler(local)
    clocks.start()
    wall0 = time.perf_counter()
    times, tri_ms = timed_loop(plan, dev_fields, args.steps)
    barrier()
    wall = time.perf_counter() - wall0
    clk = clocks.stop()
    total_ms = max_over_ranks(sum(times))
    value = world * args.steps / (total_ms / 1e3) * 3600.0

    # end to end through the C ABI from pinned host buffers
    timed_loop(plan, host_np, 1)
    barrier()
    e2e_times, _ = timed_loop(plan, host_np, args.steps)
    barrier()
    e2e_total = max_over_ranks(sum(e2e_times))
    e2e_value = world * args.steps / (e2e_total / 1e3) * 3600.0
    h2d = info["n_modes"] * info["n_planes"] * 16
    d2h = info["n_bins"] * (3 * 16 * 8 + 8)

    # the same bispectra with the triangle sums in one persistent launch
    plan.set_triangle_launch("persistent")
    timed_loop(plan, dev_fields, args.warmup)
    p_times, p_tri = timed_loop(plan, dev_fields, args.steps)
    plan.set_triangle_launch("classes")
    persistent = {"ms_per_step": float(np.mean(p_times)), "triangle_ms": float(np.mean(p_tri))}

    # latency percentiles of single jobs (device-resident and e2e)
    lat = {"p50_ms": float(np.percentile(times, 50)), "p99_ms": float(np.percentile(times, 99)),
           "e2e_p50_ms": float(np.percentile(e2e_times, 50)), "e2e_p99_ms": float(np.percentile(e2e_times, 99))}

    # mixed precision path
    mixed = None
    if not args.no_mixed:
        plan_m = beam.Plan(ctx, W["NN"], W["UL_k1"], W["LL_k1"], W["BW_k1"], Nmax=W["Nmax"], Nr=W["Nr"],
                           n_mtbin=W["n_mtbin"], precision="mixed")
        tuning["mixed"] = tune_plan(plan_m, args)
        timed_loop(plan_m, dev_fields, args.warmup)
        barrier()
        mt, mtri = timed_loop(plan_m, dev_fields, args.steps)
        barrier()
        m_total = max_over_ranks(sum(mt))
        ref = plan.run(dev_fields[0])
        got = plan_m.run(dev_fields[0])
        mixed = {"value": world * args.steps / (m_total / 1e3) * 3600.0, "unit": UNIT,
                 "ms_per_step": m_total / args.steps, "triangle_kernel_ms": float(np.mean(mtri)),
                 "speedup_vs_fp64": (sum(times) / sum(mt)), **mixed_errors(ref, got)}
        oracle_ref = oracle_fixture_bins(fields[0]) if rank == 0 else None
        if oracle_ref is not None:
            mixed["vs_oracle"] = {k: v for k, v in mixed_errors(oracle_ref, got).items()
                                  if k in ("max_rel_err", "median_rel_err", "frac_within_1e-5")}
        plan_m.close()
    else:
        oracle_ref = oracle_fixture_bins(fields[0]) if rank == 0 else None

    # int8 path: exact slice products on the int8 tensor cores (errors per (l,m,bin) against FP64 and the oracle)
    int8 = None
    if not args.no_mixed:
        plan_i = beam.Plan(ctx, W["NN"], W["UL_k1"], W["LL_k1"], W["BW_k1"], Nmax=W["Nmax"], Nr=W["Nr"],
                           n_mtbin=W["n_mtbin"], precision="int8")
        timed_loop(plan_i, dev_fields, args.warmup)
        barrier()
        it_, itri = timed_loop(plan_i, dev_fields, args.steps)
        barrier()
        i_total = max_over_ranks(sum(it_))
        ref = plan.run(dev_fields[0])
        got = plan_i.run(dev_fields[0])
        int8 = {"value": world * args.steps / (i_total / 1e3) * 3600.0, "unit": UNIT,
                "ms_per_step": i_total / args.steps, "triangle_kernel_ms": float(np.mean(itri)),
                "speedup_vs_fp64": (sum(times) / sum(it_)), **mixed_errors(ref, got),
                "launches_per_step": plan_i.refresh_info()["launches_last_run"]}
        if oracle_ref is not None:
            int8["vs_oracle"] = {k: v for k, v in mixed_errors(oracle_ref, got).items()
                                 if k in ("max_rel_err", "median_rel_err", "frac_within_1e-5")}
        plan_i.close()

    # FP64 bins against the oracle's bins of the same field (committed fixture)
    fp64_vs_oracle = None
    if oracle_ref is not None:
        e = mixed_errors(oracle_ref, plan.run(dev_fields[0]))
        fp64_vs_oracle = {"max_rel_err": e["max_rel_err"], "median_rel_err": e["median_rel_err"],
                          "bins_compared": e["bins_compared"], "counts_identical": e["counts_identical"]}

    # roofline of the dominant kernel (triangle sums on the FP64 tensor pipe, mma.sync m8n8k4.f64)
    peak = measured_fp64_peak(torch, dev)
    tri_avg = float(np.mean(tri_ms))
    flops = triangle_flops(info)
    achieved = flops / (tri_avg / 1e3) / 1e12
    roofline = {"kernel": "k_triangle<double2>", "bound": "tensor", "achieved": achieved, "peak": peak,
                "unit": "TFLOP/s", "frac": achieved / peak, "traffic": profile_traffic("k_triangle"),
                "flops_per_launch": flops, "launch_ms": tri_avg,
                "flop_basis": "8 per closed in-plane triangle term + 4 per (run, accepted triangle)",
                "peak_source": ("FP64 tensor pipe: cuBLAS DGEMM 8192^3 measured in this run "
                                "(MEASURED_PEAKS.json has no FP64 figure)")}
    if mixed is not None:
        p32 = measured_fp32_peak(torch, dev)
        a32 = flops / (mixed["triangle_kernel_ms"] / 1e3) / 1e12
        mixed["roofline"] = {"kernel": "k_triangle<float2>", "bound": "fp32", "achieved": a32, "peak": p32,
                             "unit": "TFLOP/s", "frac": a32 / p32,
                             "peak_source": "FP32 FMA: cuBLAS SGEMM 8192^3, TF32 off, measured in this run"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline_port(fields[0], info)
    batched = run_batched(ctx, args) if world == 1 and not args.no_batch else None
    serving = run_serving(ctx, args) if world == 1 and not args.no_serve else None
    field = run_field(ctx, plan, stream, args) if world == 1 and not args.no_field else None

    # kernels per bispectrum as the library counted them in the last run: mode
    # build, one triangle-sum launch per tile class, split reduction, epilogue
    per_run = plan.refresh_info()["launches_last_run"]
    gpu_launches = per_run * args.steps
    # The printed line keeps the headline numbers as top-level scalars and stays
    # short; every section in full goes to stderr as one "bench details:" line.
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD_NAME, **W, "path": "plain FP64, closed in-plane triangle sums",
                   "parallelism": f"replicas x{world} (one realization per rank per step)",
                   "l2": "flushed between steps (256 MiB write, outside the timed events)",
                   "serve_jobs": args.serve_jobs if serving else 0},
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "ms_per_step": e2e_total / args.steps},
        "clocks": clk, "gpu_launches": gpu_launches,
        "roofline": {k: roofline[k] for k in ("kernel", "bound", "achieved", "peak", "unit", "frac", "traffic")},
        "cpu_baseline": ({k: cpu[k] for k in ("value", "unit", "cores", "kind", "sample")} if cpu else None),
        "fp64_max_rel_err_vs_oracle": fp64_vs_oracle["max_rel_err"] if fp64_vs_oracle else None,
        "mixed_value": mixed["value"] if mixed else None,
        "mixed_speedup": mixed["speedup_vs_fp64"] if mixed else None,
        "mixed_max_rel_err": mixed["max_rel_err"] if mixed else None,
        "mixed_median_rel_err": mixed["median_rel_err"] if mixed else None,
        "mixed_roofline_frac": mixed["roofline"]["frac"] if mixed else None,
        "int8_value": int8["value"] if int8 else None,
        "int8_speedup": int8["speedup_vs_fp64"] if int8 else None,
        "int8_max_rel_err": int8["max_rel_err"] if int8 else None,
        "serve_jobs": args.serve_jobs if serving else 0,
        "serve_p50_ms": serving["fp64"]["p50_ms"] if serving else None,
        "serve_p99_ms": serving["fp64"]["p99_ms"] if serving else None,
        "serve_mixed_p50_ms": serving["mixed"]["p50_ms"] if serving else None,
        "serve_mixed_p99_ms": serving["mixed"]["p99_ms"] if serving else None,
        "batched_value": batched["mixed"]["batch_of_16"]["value"] if batched else None,
        "batched_fp64_value": batched["fp64"]["batch_of_16"]["value"] if batched else None,
        "batched_persistent_value": batched["mixed"]["batch_of_16_persistent"]["value"] if batched else None,
        "batched_fp64_persistent_value": batched["fp64"]["batch_of_16_persistent"]["value"] if batched else None,
        "cold_start_ms": cold["total_ms"],
        "latency_p50_ms": lat["p50_ms"], "latency_p99_ms": lat["p99_ms"],
    }
    details = {"roofline": roofline, "mixed": mixed, "int8": int8, "fp64_vs_oracle": fp64_vs_oracle, "cpu_baseline": cpu,
               "cold_start": cold, "latency": lat, "persistent_launch": persistent, "wall_s": wall, "batched": batched, "serving": serving,
               "field": field, "autotune": tuning,
               "plan": {"n_triples": info["n_triples"], "n_fourier_terms": info["n_fourier_terms"],
                        "n_run_combos": info["n_run_combos"], "plan_device_bytes": info["device_bytes"]}}
    if rank == 0:
        print("bench details: " + json.dumps(details), file=sys.stderr, flush=True)
        print(json.dumps(line), flush=True)
    plan.close()
    ctx.close()
    if world > 1:
        dist.destroy_process_group()


def run_batched(ctx, args):
    """The batched form: BATCH['realizations'] host fields through
    beam_gpu_run_batch (one launch per kernel over each batch, replayed CUDA
    graphs, host gather of batch i+1 overlapping the device work of batch i),
    timed end to end on the host clock, against the same fields one
    beam_gpu_run call at a time."""
    from barbie_b200 import beam
    from barbie_b200.synth import realization_seed, synth_field_torch
    B = BATCH
    # the field recipe on the GPU (milliseconds per field), copied to host memory
    dev = f"cuda:{ctx.device}"
    pool = [synth_field_torch(B["NN"], realization_seed(r), device=dev).cpu().numpy()
            for r in range(1, args.batch_pool + 1)]
    fields = [pool[i % len(pool)] for i in range(B["realizations"])]
    out = {"workload": f"{B['realizations']} realizations at NN={B['NN']}, Nmax={B['Nmax']}, Nr={B['Nr']}, "
                       f"k1 bins 1..{B['UL_k1']} width 1",
           "fields": (f"{len(pool)} distinct seeded fields (seeds 100020+146r, r=1..{len(pool)}; the field recipe "
                      f"run with torch on the GPU, then held in host memory)"
                      + (f", cycled over the {B['realizations']} realizations" if len(pool) < B["realizations"] else "")),
           "timing": "host wall clock around each call (host gather, H2D, kernels, D2H of the bins)"}
    for prec in ("mixed", "fp64"):
        plan = beam.Plan(ctx, B["NN"], B["UL_k1"], B["LL_k1"], B["BW_k1"], Nmax=B["Nmax"], Nr=B["Nr"],
                         n_mtbin=B["n_mtbin"], precision=prec)
        res = {}
        for mode in ("classes", "persistent"):
            plan.set_triangle_launch(mode)
            for label, batch in (("batched", 0), ("batch_of_16", 16)):
                plan.run_batch(fields, batch=batch)  # warm-up: slots and graphs
                t = []
                for _ in range(max(1, args.steps // 3)):
                    t0 = time.perf_counter()
                    plan.run_batch(fields, batch=batch)
                    t.append(time.perf_counter() - t0)
                key = label if mode == "classes" else f"{label}_persistent"
                res[key] = {"value": len(fields) / min(t) * 3600.0, "seconds_per_call": min(t),
                            "launches_per_batch": plan.refresh_info()["launches_last_run"]}
        plan.set_triangle_launch("classes")
        for f in pool[:2]:
            plan.run(f)
        t0 = time.perf_counter()
        for f in fields:
            plan.run(f)
        res["one_at_a_time"] = {"value": len(fields) / (time.perf_counter() - t0) * 3600.0}
        res["unit"] = UNIT
        res["batch_speedup"] = res["batched"]["value"] / res["one_at_a_time"]["value"]
        res["device_bytes"] = plan.refresh_info()["device_bytes"]
        out[prec] = res
        plan.close()
    return out


def tune_plan(plan, args):
    """beam_gpu_plan_autotune on the plan (work decomposition of the triangle
    sums chosen by timing on this device), or None with --no-autotune."""
    if args.no_autotune:
        return None
    t0 = time.perf_counter()
    rep = plan.autotune(reps=3)
    rep["seconds"] = time.perf_counter() - t0
    tau0 = 1024 if plan.precision == "fp64" else 512  # the library's defaults
    default = [c for c in rep["candidates"] if c["tau0"] == tau0 and c["balance"] == 8.0]
    if default:
        rep["default_ms"] = default[0]["ms"]
    return rep


def run_field(ctx, plan, stream, args):
    """On-device field ingestion at the bench's NN: the reference generator
    (beam_gpu_field_generate: fill, 3 backward passes, variance, 3 forward
    passes) and a real-space cube to the r2c buffer (beam_gpu_field_ingest: 3
    forward passes), both device-resident, timed with CUDA events on the
    library's stream around each call; and a job from a real-space cube on the
    device to its bins (ingest + beam_gpu_run). Every buffer (455 MB) exceeds L2.
    Roofline: each FFT pass reads and writes the half-complex array once,
    2 x 16 NN^2 (NN/2+1) bytes; achieved = passes x that / call time."""
    import torch
    from barbie_b200 import beam
    NN = WORKLOAD["NN"]
    dev = torch.device("cuda", ctx.device)
    tiles = None if args.no_autotune else beam.field_autotune(ctx, NN)
    out = torch.empty((NN, NN, NN + 2), dtype=torch.float64, device=dev)
    cube = torch.randn((NN, NN, NN), dtype=torch.float64, device=dev,
                       generator=torch.Generator(device=dev).manual_seed(11))
    reps = max(3, min(args.steps, 10))

    def timed(fn):
        for _ in range(2):
            fn()
        ms = []
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            fn()
            e1.record(stream)
            e1.synchronize()
            ms.append(e0.elapsed_time(e1))
        return float(np.median(ms))

    gen_ms = timed(lambda: beam.generate_field(ctx, NN, beam.field_seed(1), out=out))
    gen_launches = ctx.field_launches()
    ing_ms = timed(lambda: beam.ingest_field(ctx, cube, out=out))
    ing_launches = ctx.field_launches()
    job_ms = timed(lambda: (beam.ingest_field(ctx, cube, out=out), plan.run(out)))
    # power spectrum multipoles of the device buffer (calpow_mom): one read of the buffer
    pk_ms = timed(lambda: beam.power_multipoles(ctx, out, NN, LL=0.56, Nbin=10))
    pk_bytes = 16 * NN * NN * (NN // 2 + 1)
    pass_bytes = 2 * 16 * NN * NN * (NN // 2 + 1)
    peak = hbm_peak()
    ach = 3 * pass_bytes / (ing_ms / 1e3) / 1e9
    del out, cube
    torch.cuda.empty_cache()
    return {"workload": f"NN={NN} r2c buffer double[{NN}][{NN}][{NN + 2}]; generator constants LL=0.56, ff=0.5, "
                        "beta=1 (generate_field.c:45-50)",
            "generate_ms": gen_ms, "generate_launches": gen_launches,
            "ingest_ms": ing_ms, "ingest_launches": ing_launches,
            "cube_to_bins_ms": job_ms, "cube_to_bins_per_hour": 3600e3 / job_ms,
            "roofline": {"kernel": "k_fft_rows_r2c + k_fft_cols (3 passes of one ingestion)", "bound": "hbm",
                         "achieved": ach, "peak": peak[0], "unit": "GB/s", "frac": ach / peak[0],
                         "bytes_per_pass": pass_bytes, "peak_source": peak[1]},
            "timing": "median of CUDA-event times around each call on the library stream",
            "autotune": tiles,
            "power_multipoles": {"ms": pk_ms, "bins": 10, "roofline": {
                "kernel": "k_pk_rows + k_pk_total", "bound": "hbm", "achieved": pk_bytes / (pk_ms / 1e3) / 1e9,
                "peak": peak[0], "unit": "GB/s", "frac": pk_bytes / (pk_ms / 1e3) / 1e9 / peak[0],
                "bytes": pk_bytes}}}


def hbm_peak():
    """(GB/s, source) of the measured HBM copy bandwidth."""
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as fh:
            return float(json.load(fh)["hbm_gbs"]), "MEASURED_PEAKS.json hbm_gbs (measured copy)"
    except (OSError, ValueError, KeyError):
        return 6650.0, "fallback 6.65 TB/s (no measured figure)"


def run_serving(ctx, args):
    """The serving form: a Poisson stream of jobs, each one realization with NN
    drawn from SERVE, bins of width 1 or 2, through the job server (admission
    by device-memory footprint, up to 4 jobs on the device at once). Reports
    per-job latency (submission to bins on the host) and throughput, for the
    plain and the mixed path."""
    from barbie_b200 import beam
    from barbie_b200.synth import realization_seed, synth_field
    rng = np.random.default_rng(500)
    nns = sorted(SERVE)
    pool = {NN: synth_field(NN, realization_seed(1000 + NN)) for NN in nns}
    jobs = [(int(rng.choice(nns)), int(rng.choice([1, 2]))) for _ in range(args.serve_jobs)]
    gaps = rng.exponential(1.0, size=len(jobs))  # unit-mean gaps, scaled to the rate below
    out = {"workload": f"{len(jobs)} jobs per path, NN uniform over {nns}, (Nmax, Nr) = "
                       f"{ {k: v for k, v in SERVE.items()} }, k1 bins 1..Nmax width 1 or 2, 5 t x 5 mu bins",
           "arrivals": "Poisson at 70% of the mean single-job service rate measured in the warm-up "
                       "(first job per configuration, plan creation included)",
           "fields": "one seeded field per NN (job r2c buffers are read from host memory per job)",
           "latency": "submission to bins in host memory, host clock"}
    for prec in ("fp64", "mixed"):
        srv = beam.Server(ctx, max_active=4)
        service = {}
        for NN, BW in sorted(set(jobs)):  # warm-up: builds and caches the plans, one job per configuration
            Nmax, Nr = SERVE[NN]
            j = srv.submit(pool[NN], NN, Nmax + 1, 1, BW, Nmax=Nmax, Nr=Nr, precision=prec)
            info = srv.wait(j, 600000)
            srv.take(j)
            service[(NN, BW)] = info["run_ms"] / 1e3
        cached = {}
        for NN, BW in sorted(set(jobs)):  # the same jobs again, plans cached: device work alone
            Nmax, Nr = SERVE[NN]
            j = srv.submit(pool[NN], NN, Nmax + 1, 1, BW, Nmax=Nmax, Nr=Nr, precision=prec)
            info = srv.wait(j, 600000)
            srv.take(j)
            cached[(NN, BW)] = info["run_ms"]
        mean_service = float(np.mean([service[k] for k in jobs]))
        rate = 0.7 / mean_service
        ids = []
        t0 = time.perf_counter()
        t_next = t0
        for (NN, BW), g in zip(jobs, gaps):
            t_next += g / rate
            dt = t_next - time.perf_counter()
            if dt > 0:
                time.sleep(dt)
            Nmax, Nr = SERVE[NN]
            ids.append(srv.submit(pool[NN], NN, Nmax + 1, 1, BW, Nmax=Nmax, Nr=Nr, precision=prec))
        lat, run = [], []
        for j in ids:
            info = srv.wait(j, 600000)
            srv.take(j)
            lat.append(info["total_ms"])
            run.append(info["run_ms"])
        wall = time.perf_counter() - t0
        _, peak = srv.memory()
        srv.close()
        out[prec] = {"p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
                     "max_ms": float(np.max(lat)), "service_p50_ms": float(np.percentile(run, 50)),
                     "throughput": len(jobs) / wall * 3600.0, "unit": UNIT, "arrival_rate_per_s": rate,
                     "mean_service_alone_s": mean_service, "peak_device_bytes": peak,
                     "service_alone_ms": {f"NN{k[0]}_BW{k[1]}": v * 1e3 for k, v in sorted(service.items())},
                     "service_cached_ms": {f"NN{k[0]}_BW{k[1]}": v for k, v in sorted(cached.items())}}
    return out


def cpu_baseline_port(field, info):
    """The oracle (CPU restatement of the reference) timed on a bounded random
    sample of accepted triangles, transforms and pixel sums over all host cores,
    extrapolated to one full bispectrum."""
    from oracle import oracle_py
    W = WORKLOAD
    cores = os.cpu_count() or 1
    ntri = info["n_triples"]
    nsample = int(min(ntri, 1500 * cores))
    rng = np.random.default_rng(2024)
    sample = np.sort(rng.choice(ntri, size=nsample, replace=False))
    r = oracle_py.time_sample(field, W["NN"], W["Nmax"], W["Nr"], W["UL_k1"], W["LL_k1"], W["BW_k1"], sample, cores)
    n_arrays = W["Nmax"] * W["Nr"]  # wrapid_fast builds every (plane, ring) array
    secs = ntri * r["t_sum"] / nsample + n_arrays * r["t_fft"] / max(1, r["n_fft"])
    return {"value": 3600.0 / secs, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"{nsample} random accepted triangles of {ntri} (pixel sums) and the {r['n_fft']} plane-ring "
                      f"transforms they need, extrapolated to {ntri} triangles and {n_arrays} transforms",
            "sample_seconds": r["t_sum"] + r["t_fft"], "seconds_per_bispectrum": secs}


# --------------------------------------------------------------- reference
def reference_full_run_check(ref_bin, cores):
    """A whole reference run at a small configuration (barbie 96 1 21 1 1 with
    Nmax=32, Nr=20), timed, beside the per-triangle extrapolation the arm uses
    at NN=384 applied to the same configuration (windows of ring triplets of
    one p1, one process at a time): how far the extrapolated triangle-loop
    time is from the measured one."""
    from oracle import oracle_py
    from barbie_b200.synth import realization_seed, synth_field, write_field
    NN, Nmax, Nr, UL, LL, BW = 96, 32, 20, 21, 1, 1
    scratch = tempfile.mkdtemp(prefix="beam_refcheck_")
    try:
        os.makedirs(os.path.join(scratch, f"ResFiles_N{NN}", "data_files"), exist_ok=True)
        write_field(os.path.join(scratch, f"field_N{NN}_R1.txt"), synth_field(NN, realization_seed(1)))
        env = dict(os.environ, BEAM_REF_NMAX=str(Nmax), BEAM_REF_NR=str(Nr), BEAM_REF_NTHREADS=str(cores))

        def run(extra):
            out = subprocess.run(["bash", "-c", f"ulimit -s unlimited; exec {ref_bin} {NN} 1 {UL} {LL} {BW}"],
                                 cwd=scratch, env=dict(env, **extra), capture_output=True, text=True)
            m = re.search(r"Total time ([0-9.]+)", out.stdout)
            return float(m.group(1)) if m else None

        full = run({})  # builds the caches, then the whole triangle loop
        rings = oracle_py.closed_rings(NN, Nr, Nmax)
        tri, _ = oracle_py.enumerate_triples(NN, Nmax, Nr, UL, LL, BW, rings4=rings)
        per_tri = []
        for p1 in sorted(set(int(v) for v in tri["p1"]))[::4]:
            counts = np.bincount(tri["rp"][tri["p1"] == p1], minlength=len(rings))
            n = int(counts.sum())
            t = run({"BEAM_REF_P1_LO": str(p1), "BEAM_REF_P1_HI": str(p1 + 1)}) if n else None
            if t and t > 0:
                per_tri.append(t / n)
        pred = len(tri) * float(np.median(per_tri)) if per_tri else None
        return {"workload": f"barbie {NN} 1 {UL} {LL} {BW}, Nmax={Nmax}, Nr={Nr}", "triangles": int(len(tri)),
                "measured_loop_s": full, "extrapolated_loop_s": pred,
                "extrapolated_over_measured": (pred / full) if (pred and full) else None,
                "samples": f"{len(per_tri)} single-p1 runs, one process at a time"}
    finally:
        shutil.rmtree(scratch, ignore_errors=True)


def run_reference(args):
    world, rank, _ = dist_setup(args)
    if rank != 0:
        return
    from oracle import oracle_py
    ref_bin = oracle_py.REF_BIN
    if not os.path.exists(ref_bin):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/barbie_ref was not built (reference "
                          "sources absent when building)"}), flush=True)
        return
    from barbie_b200.synth import realization_seed, synth_field, write_field
    W = WORKLOAD
    NN = W["NN"]
    cores = os.cpu_count() or 1
    scratch = os.path.join(ROOT, "_bench_ref")
    os.makedirs(os.path.join(scratch, f"ResFiles_N{NN}", "data_files"), exist_ok=True)
    field_path = os.path.join(scratch, f"field_N{NN}_R1.txt")
    if not os.path.exists(field_path):
        write_field(field_path, synth_field(NN, realization_seed(1)))
    # Nthreads (barbie.c:68, the FFTW threads of its cache build) set to the host's cores
    env = dict(os.environ, BEAM_REF_NMAX=str(W["Nmax"]), BEAM_REF_NR=str(W["Nr"]), BEAM_REF_NTHREADS=str(cores))

    def ref_cmd(p1lo, p1hi, rplo, rphi):
        e = dict(env, BEAM_REF_P1_LO=str(p1lo), BEAM_REF_P1_HI=str(p1hi), BEAM_REF_RP_LO=str(rplo),
                 BEAM_REF_RP_HI=str(rphi))
        args_ = f"ulimit -s unlimited; exec {ref_bin} {NN} 1 {W['UL_k1']} {W['LL_k1']} {W['BW_k1']}"
        return ["bash", "-c", args_], e

    # set-up: the reference's own caches (closed_rings_<NN> and the plane-ring files)
    cmd, e = ref_cmd(0, 0, 0, 0)
    t0 = time.perf_counter()
    out = subprocess.run(cmd, cwd=scratch, env=e, capture_output=True, text=True)
    t_setup = time.perf_counter() - t0
    m = re.search(r"4\. Calculation done successfully \(in ([0-9.]+) sec\)", out.stdout)
    t_cache = float(m.group(1)) if m else t_setup
    m = re.search(r"2\. Calculation of ring combinations completed successfully \(in ([0-9.]+) sec\)", out.stdout)
    t_calcr = float(m.group(1)) if m else 0.0

    # samples: consecutive ring triplets of one p1, about `target` accepted triangles each
    rings = oracle_py.closed_rings(NN, W["Nr"], W["Nmax"])
    tri, _ = oracle_py.enumerate_triples(NN, W["Nmax"], W["Nr"], W["UL_k1"], W["LL_k1"], W["BW_k1"], rings4=rings)
    ntri = len(tri)
    nproc = max(1, min(cores, 64))
    target = 4000
    # every window holds min(target, all of its p1's) accepted triangles: a start
    # too close to the end of the triplet list moves back, so no process runs a
    # window of a few triangles that start-up would dominate, or of none
    samples = []
    per_p1 = {p1: np.bincount(tri["rp"][tri["p1"] == p1], minlength=len(rings)) for p1 in np.unique(tri["p1"])}
    p1s = [p1 for p1 in sorted(per_p1) if per_p1[p1].sum() > 0]
    for k in range(nproc * max(1, args.steps + args.warmup)):
        p1 = int(p1s[(7 * k) % len(p1s)])
        counts = per_p1[p1]
        cum = np.concatenate([[0], np.cumsum(counts)])
        want = min(target, int(cum[-1]))
        start = (k * 131) % len(rings)
        start = min(start, int(np.searchsorted(cum, cum[-1] - want, side="right")) - 1)  # suffix holds >= want
        end = int(np.searchsorted(cum, cum[start] + want, side="left"))
        samples.append((p1, start, end, int(cum[end] - cum[start])))

    def step(k0):
        procs = []
        for j in range(nproc):
            p1, a, b, n = samples[(k0 * nproc + j) % len(samples)]
            cmd, e = ref_cmd(p1, p1 + 1, a, b)
            procs.append((subprocess.Popen(cmd, cwd=scratch, env=e, stdout=subprocess.PIPE, stderr=subprocess.STDOUT,
                                           text=True), n))
        rates = []
        for pr, n in procs:
            o, _ = pr.communicate()
            m = re.search(r"Total time ([0-9.]+)", o)
            if m and float(m.group(1)) > 0 and n > 0:
                rates.append(n / float(m.group(1)))
        return rates

    for k in range(args.warmup):
        step(k)
    vals, per_tri = [], []
    for k in range(args.steps):
        rates = step(args.warmup + k)
        # each process is one realization stream: per bispectrum the loop over all
        # accepted triangles plus the cache build it needs
        per = [ntri / r + t_cache + t_calcr for r in rates]
        vals.append(sum(3600.0 / s for s in per))
        per_tri.extend(1.0 / r for r in rates)
    value = float(np.mean(vals))
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD_NAME, **W},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": nproc, "kind": "reference",
                             "sample": f"{nproc} concurrent reference processes per step, each the triangle loop "
                                       f"of one p1 over a window of ring triplets (~{target} accepted triangles); "
                                       f"extrapolated to {ntri} triangles plus the measured cache build "
                                       f"({t_cache:.1f} s) and calCR ({t_calcr:.1f} s)",
                             "seconds_per_triangle": float(np.median(per_tri)) if per_tri else None,
                             # one reference process for a whole bispectrum (its triangle loop is single-threaded)
                             "one_process": ({"bispectra_per_hour": 3600.0 / (ntri * float(np.median(per_tri)) + t_cache + t_calcr),
                                              "seconds_per_bispectrum": ntri * float(np.median(per_tri)) + t_cache + t_calcr}
                                             if per_tri else None)},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    try:
        line["cpu_baseline"]["full_run_check"] = reference_full_run_check(ref_bin, cores)
    except (OSError, subprocess.SubprocessError, ValueError) as e:
        line["cpu_baseline"]["full_run_check"] = {"error": str(e)}
    print(json.dumps(line), flush=True)
    shutil.rmtree(scratch, ignore_errors=True)  # the reference's disk caches: ~9.4 GB at NN=384


def main():
    args = parse_args()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
