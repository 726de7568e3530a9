#!/usr/bin/env python
"""Benchmark of the multi-stage quantum-walk hot path.

Metric: instances/s at n = 20, m = 4 — one instance is the reference's full
per-problem job (MultiQW.cpp:296-455): the Ising diagonal, the stage
schedule, and 100 time samples x 4 stages of Chebyshev/Clenshaw propagation
of a 2^20-amplitude state, reduced to the mean ground-state probability.

A step is one batch of `--batch` seeded synthetic Sherrington–Kirkpatrick
instances (J_ij, h_i ~ N(0,1), the reference's file layout; the reference's
datasets are not used). `value` times the device path with the batch already
resident in device memory (mqw_plan_execute); `e2e` times the public C ABI
call from host buffers (mqw_run_problems: upload, schedule, run, read-back).
L2 is flushed (256 MB write) between timed steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

With --impl reference the line times the reference's own CPU hot loop
(Clenshaw_step, compiled from the reference source into oracle/_ref) driven
by the oracle's restatement of its problem loop, run-script style (one
process per core), on a bounded sample of the same workload.
"""
from __future__ import annotations

import argparse
import json
import multiprocessing as mp
import os
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = ("instances/s at n=20,m=4 (|ΔP|≤1e-5 vs FP64); "
          "mean P_gs learned vs heuristic")
BYTES_PER_TERM_AMP = {"fp32": 36, "fp64": 72}  # algorithmic, see DESIGN.md
PEAKS_FALLBACK = {"hbm_gbs": 6650.0}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="mqw", choices=["mqw", "reference"])
    ap.add_argument("--n", type=int, default=20)
    ap.add_argument("--m", type=int, default=4)
    ap.add_argument("--batch", type=int, default=2, help="instances per step per GPU")
    ap.add_argument("--samples", type=int, default=100)
    ap.add_argument("--precision", default="fp32", choices=["fp32", "fp64"])
    ap.add_argument("--group", type=int, default=0)
    ap.add_argument("--seed", type=int, default=20)
    ap.add_argument("--no-check", action="store_true", help="skip the FP64 |dP| check")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline")
    ap.add_argument("--cpu-samples", type=int, default=2, help="samples per CPU worker")
    return ap.parse_args()


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return d, "measured"
    return PEAKS_FALLBACK, "fallback"


# ---- clocks -------------------------------------------------------------------

class ClockSampler:
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_id: str):
        self.proc = None
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", gpu_id, f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None

    def stop(self):
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
            out, _ = self.proc.communicate()
        rows = []
        for line in out.strip().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 8:
                continue
            try:
                rows.append((float(parts[0]), float(parts[1]), parts[4:8]))
            except ValueError:
                continue
        if not rows:
            return None
        load = [r for r in rows if r[0] > 0.5 * r[1]] or rows
        sm = sorted(r[0] for r in load)
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i, v in enumerate(r[2]) if v.lower() == "active"})
        return {"sm_mhz": sm[len(sm) // 2], "sm_max_mhz": max(r[1] for r in rows),
                "reasons": reasons, "samples": len(rows)}


def gpu_selector(torch, dev):
    try:
        u = str(torch.cuda.get_device_properties(dev).uuid)
        return u if u.startswith("GPU-") else "GPU-" + u
    except Exception:
        vis = os.environ.get("CUDA_VISIBLE_DEVICES")
        return vis.split(",")[dev] if vis else str(dev)


# ---- CPU baseline (reference hot loop, one process per core) ------------------

def _cpu_worker(args):
    n, m, seed, samples = args
    sys.path.insert(0, ROOT)
    from oracle import oracle as O
    raw = O.sk_instances(n, 1, seed)
    use_ref = O.ref_lib() is not None
    t0 = time.perf_counter()
    O.run_problems(n, m, raw, 1, samples, "f32", use_ref_step=use_ref)
    return time.perf_counter() - t0, use_ref


def cpu_baseline(n, m, seed, samples_per_worker, workers=None):
    cores = len(os.sched_getaffinity(0))
    workers = workers or cores
    ctx = mp.get_context("spawn")
    jobs = [(n, m, seed + i, samples_per_worker) for i in range(workers)]
    t0 = time.perf_counter()
    with ctx.Pool(workers) as pool:
        res = pool.map(_cpu_worker, jobs)
    wall = time.perf_counter() - t0
    busy = max(r[0] for r in res)
    kind = "reference" if all(r[1] for r in res) else "port"
    inst = workers * samples_per_worker / 100.0
    return {
        "value": inst / busy, "unit": "instances/s", "cores": workers, "kind": kind,
        "sample": (f"{workers} processes x {samples_per_worker} of the 100 samples of one "
                   f"n={n}, m={m} instance each (FP32; "
                   + ("reference Clenshaw_step, MultiQW.cpp:88-173, AVX-512 build" if kind == "reference"
                      else "oracle restatement") + "); instances/s = samples/100 / slowest worker"),
        "wall_s": wall,
    }


# ---- main ---------------------------------------------------------------------

def main():
    a = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if a.impl == "reference":
        if rank != 0:
            return
        times = []
        base = None
        for step in range(a.warmup + a.steps):
            b = cpu_baseline(a.n, a.m, a.seed + 1000 * step, 1)
            if step >= a.warmup:
                times.append(b)
            base = b
        val = sum(t["value"] for t in times) / len(times)
        line = {
            "metric": METRIC, "value": val, "unit": "instances/s", "n_gpus": a.gpus,
            "steps": a.steps, "warmup": a.warmup, "ms_per_step": 1000.0 / val,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic seeded SK instances (J,h ~ N(0,1))",
            "impl": "reference",
            "config": {"workload": f"sk_n{a.n}_m{a.m}", "n": a.n, "m": a.m, "samples": 100},
            "cpu_baseline": {k: base[k] for k in ("kind", "cores", "sample")} | {"value": val, "unit": "instances/s"},
            "e2e": {"value": val, "unit": "instances/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        }
        print(json.dumps(line))
        return

    import numpy as np
    import torch
    import torch.distributed as dist

    import multistageqw_b200 as M

    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=600))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    ctx = M.Context(local)
    stream = torch.cuda.current_stream(dev)
    raw = M.sk_instances(a.n, a.batch, a.seed + 7919 * rank)
    plan = M.Plan(ctx, a.n, a.m, raw, samples=a.samples, precision=a.precision, group=a.group)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize(dev)

    for _ in range(a.warmup):
        plan.execute(stream.cuda_stream)
    barrier()
    clocks = ClockSampler(gpu_selector(torch, local))
    step_ms = []
    kern_ms = []
    term_amps = 0.0
    launches = 0
    term_launches = 0
    for _ in range(a.steps):
        flush.zero_()
        torch.cuda.synchronize(dev)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        plan.execute(stream.cuda_stream)
        e1.record(stream)
        torch.cuda.synchronize(dev)
        step_ms.append(e0.elapsed_time(e1))
        st = plan.stats()
        kern_ms.append(st["kernel_ms"])
        term_amps += st["term_amps"]
        launches += st["launches"]
        term_launches += st["term_launches"]
    barrier()
    clk = clocks.stop()
    total_ms = sum(step_ms)
    if world > 1:
        t = torch.tensor([total_ms], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
    value = world * a.batch * a.steps / (total_ms / 1000.0)

    # End to end through the public API from pinned host buffers.
    raw_pinned = torch.from_numpy(np.ascontiguousarray(raw)).pin_memory().numpy()
    e2e_ms = []
    h2d = d2h = 0.0
    for i in range(max(1, min(a.steps, 2))):
        flush.zero_()
        barrier()
        t0 = time.perf_counter()
        r = ctx.run_problems(a.n, a.m, raw_pinned, samples=a.samples, precision=a.precision, group=a.group)
        torch.cuda.synchronize(dev)
        e2e_ms.append((time.perf_counter() - t0) * 1000.0)
        h2d, d2h = r["stats"]["h2d_bytes"], r["stats"]["d2h_bytes"]
    e2e_total = sum(e2e_ms)
    if world > 1:
        t = torch.tensor([e2e_total], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_total = float(t.item())
    e2e_val = world * a.batch * len(e2e_ms) / (e2e_total / 1000.0)

    # |dP| of the timed FP32 results against the FP64 path (first instance).
    check = None
    res = plan.results()
    if not a.no_check and a.precision == "fp32":
        r64 = ctx.run_problems(a.n, a.m, raw[:1], samples=a.samples, precision="fp64", group=a.group)
        check = {"max_abs_dP_vs_fp64": float(abs(res["p"][0] - r64["p"][0])),
                 "instances_checked": 1, "p_fp32": float(res["p"][0]), "p_fp64": float(r64["p"][0])}

    pk, pk_kind = peaks()
    kms = sum(kern_ms)
    achieved = BYTES_PER_TERM_AMP[a.precision] * term_amps / (kms / 1000.0) / 1e9 if kms > 0 else None
    peak = pk["hbm_gbs"]
    roofline = {
        "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
        "frac": achieved / peak if achieved else None, "traffic": None,
        "peak_source": f"hbm_gbs of {pk_kind}",
        "kernel": "term_kernel (grid-path Clenshaw term)",
        "bytes_per_launch": BYTES_PER_TERM_AMP[a.precision] * term_amps / max(1, term_launches),
        "avg_launch_us": 1000.0 * kms / max(1, term_launches),
    }

    line = None
    if rank == 0:
        cpu = None
        if world == 1 and not a.no_cpu:
            try:
                cpu = cpu_baseline(a.n, a.m, 4242, a.cpu_samples)
            except Exception as ex:  # the baseline is reported, not required
                cpu = {"value": None, "error": str(ex)}
        line = {
            "metric": METRIC, "value": value, "unit": "instances/s", "n_gpus": world,
            "steps": a.steps, "warmup": a.warmup, "ms_per_step": total_ms / a.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32" if a.precision == "fp32" else "f64",
            "data": "synthetic seeded SK instances (J,h ~ N(0,1)); reference datasets not used",
            "config": {"workload": f"sk_n{a.n}_m{a.m}", "n": a.n, "m": a.m,
                       "instances_per_step": a.batch * world, "samples": a.samples,
                       "precision": a.precision, "group": a.group or "auto",
                       "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                       "l2": "flushed between timed steps (256 MB write)"},
            "e2e": {"value": e2e_val, "unit": "instances/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h},
            "gpu_launches": launches // max(1, a.steps),
            "roofline": roofline,
            "cpu_baseline": cpu,
            "clocks": clk,
            "check": check,
            "results_head": [float(x) for x in res["p"][:4]],
        }
        print(json.dumps(line), flush=True)
    plan.close()
    ctx.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
