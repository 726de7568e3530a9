#!/usr/bin/env python
"""Benchmark of the multi-stage quantum-walk hot path.

Metric: instances/s at n = 20, m = 4 — one instance is the reference's full
per-problem job (MultiQW.cpp:296-455): the Ising diagonal, the stage
schedule, and 100 time samples x 4 stages of Chebyshev/Clenshaw propagation
of a 2^20-amplitude state, reduced to the mean ground-state probability.

A step is one batch of `--batch` seeded synthetic Sherrington–Kirkpatrick
instances (J_ij, h_i ~ N(0,1), the reference's file layout; the reference's
datasets are not used). `value` times the device path with the batch already
resident in device memory (mqw_plan_execute; after the first execution this
replays a CUDA graph of the whole device pipeline); `e2e` times the public C
ABI from host buffers (plan create: upload and host schedule; execute;
read-back). L2 is flushed (256 MB write) between timed steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Other workloads (--workload): adam_n20_m4 (the headline's shape on the
reference's own instances: the first --batch of data/AdamData/SK_20n, a
committed byte copy), mixed (a seeded subset of the mixed n=12..20, m=2..5
batch), n28 (one n=28, m=3 instance, a few samples per step), mixed_full (the
whole 4096-instance mixed batch as one plan; one JSON report) and precision
(the n=24 near-degenerate FP32/FP64/CPU study; one JSON report).

With --impl reference the line times the reference's own CPU hot loop
(Clenshaw_step, compiled from the reference source into oracle/_ref) driven
by the oracle's restatement of its problem loop, run-script style (one
process per core): every timed step is one whole instance of the workload
(its 100 samples split into contiguous ranges over the processes); n = 28
times terms of the reference's step and scales them (a whole instance takes
hours per core); the mixed workload runs the first samples of every
instance.

roofline: the dominant kernel — pass_kernel, or real_pass_kernel when the
shared-basis chains carry more bytes than the walks' passes (the headline:
with the product bases no walk runs a recurrence) — timed alone (CUDA events
around a pass-only replay in the plan's tuned shape) against the tier that
holds its working set — L2 (the library's own L2 copy probe) when the walks in
flight fit, else HBM (MEASURED_PEAKS.json); frac = bytes_per_launch /
avg_launch_us / peak.
"""
from __future__ import annotations

import argparse
import json
import multiprocessing as mp
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = ("instances/s at n=20,m=4 (|ΔP|≤1e-5 vs FP64); "
          "mean P_gs learned vs heuristic")
BYTES_PER_TERM_AMP = {"fp32": 36, "fp32c": 36, "fp64": 72}  # algorithmic bytes per term·amp
PEAKS_FALLBACK = {"hbm_gbs": 6650.0}
# DRAM bytes (read + write) per term·amp of one pass_kernel launch from an
# ncu capture of the workload (cold caches: ncu flushes them between
# replays), keyed by config.workload: n = 20, 29.40 MB per 2^20-amplitude
# launch; n = 24 and n = 28 (2^12 single-CTA tiles with global axes), the
# same pass shape captured on an n = 26 walk (6 global axes), 1880.3 +
# 1050.6 MB per 2^26-amplitude launch, per amplitude.
DRAM_BYTES_PER_TERM_AMP = {"sk_n20_m4": 29.40e6 / 2**20, "adam_sk20n_m4": 29.40e6 / 2**20,
                           "sk_n24_m4": 2930.9e6 / 2**26, "sk_n28_m3_seed7": 2930.9e6 / 2**26}
# The real chain pass (shared-basis chains, FP32): algorithmic bytes per
# amplitude (read b_{r+1}, b_{r+2} and D, write b_r) and cold-cache DRAM
# bytes per amplitude of one launch from an ncu capture, keyed by workload.
CHAIN_BYTES_PER_AMP = 16
# profiles/real_pass_kernel_sk_n20_m4.md: 12.63 MB read, 0 written per
# launch of 2^20 amplitudes (the read set b_{r+1}, P, D).
CHAIN_DRAM_BYTES_PER_AMP = {"sk_n20_m4": 12.62592e6 / 2**20, "adam_sk20n_m4": 12.62592e6 / 2**20}
# L1 data-pipe (LSU) wavefronts of one n = 20 chain launch (2^12 tiles, 256
# threads), the mean of a tiling-1 and a tiling-2 launch (705 028 and
# 869 270, profiles/real_pass_kernel_sk_n20_m4.md); the pipe takes one
# wavefront per cycle per SM.
CHAIN_L1_WAVEFRONTS_PER_AMP = {20: 787149.0 / 2**20}
# Host memory the CPU legs may use at once (all worker processes together).
CPU_MEM_BUDGET = 24 << 30


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="mqw", choices=["mqw", "reference"])
    ap.add_argument("--workload", default="sk_n20_m4",
                    choices=["sk_n20_m4", "adam_n20_m4", "mixed", "n28", "precision",
                             "mixed_full"])
    ap.add_argument("--n", type=int, default=20)
    ap.add_argument("--m", type=int, default=4)
    ap.add_argument("--batch", type=int, default=2, help="instances per step per GPU")
    ap.add_argument("--samples", type=int, default=100)
    ap.add_argument("--precision", default="fp32", choices=["fp32", "fp64", "fp32c"])
    ap.add_argument("--group", type=int, default=0, help="walks per launch (0: autotuned)")
    ap.add_argument("--tile-log", type=int, default=0, help="grid-path tile cap (0: autotuned)")
    ap.add_argument("--lanes", type=int, default=0, help="concurrent launch lanes (0: autotuned)")
    ap.add_argument("--threads", type=int, default=0, help="CTA threads 512/256 (0: autotuned)")
    ap.add_argument("--lane-smem", type=int, default=0, help="lane axes: 1 shared memory, -1 shuffles")
    ap.add_argument("--tma", type=int, default=0,
                    help="tile staging: 1 bulk copies, 2 second exchange tile, -1 cp.async")
    ap.add_argument("--cluster", type=int, default=0,
                    help="widest tile with axes left over: 1 cluster, -1 global axes (0: autotuned)")
    ap.add_argument("--seed", type=int, default=20)
    ap.add_argument("--no-check", action="store_true", help="skip the FP64 |dP| check")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline")
    ap.add_argument("--cpu-walks", type=int, default=4, help="precision: CPU-checked instances")
    return ap.parse_args()


def find_key(d, key):
    """The first value stored under `key` anywhere in a nested dict/list."""
    if isinstance(d, dict):
        if key in d:
            return d[key]
        d = list(d.values())
    if isinstance(d, list):
        for v in d:
            r = find_key(v, key)
            if r is not None:
                return r
    return None


def peaks():
    """HBM copy bandwidth for the roofline: the measured figure of this pool's
    B200s (MEASURED_PEAKS.json, written beside this file by the pool), else
    the pool's earlier measurement."""
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        try:
            with open(p) as f:
                v = find_key(json.load(f), "hbm_gbs")
            if isinstance(v, (int, float)) and v > 0:
                return {"hbm_gbs": float(v)}, "measured"
        except (OSError, ValueError):
            pass
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
        return self.summarize(out)

    @staticmethod
    def summarize(out: str):
        """Median SM clock under load, the maximum, and every throttle reason
        seen active, from nvidia-smi's CSV lines (FIELDS order, no units)."""
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


# ---- CPU baselines (reference hot loop, one process per core) ------------------

def _cpu_range_worker(args):
    """Samples [s0, s1) of one instance through the reference pipeline (the
    reference's own Clenshaw_step when the partial build is present)."""
    n, m, raw, s0, s1 = args
    sys.path.insert(0, ROOT)
    from oracle import oracle as O
    use_ref = O.ref_lib() is not None
    t0 = time.perf_counter()
    ps, _ = O.run_sample_range(n, m, raw, s0, s1, "f32", use_ref_step=use_ref)
    return ps, time.perf_counter() - t0, use_ref


def sample_ranges(samples: int, workers: int):
    """run.sh's split of a problem range over processes (run.sh:27-38),
    applied to one instance's samples: contiguous ranges, the first
    `samples % workers` one longer."""
    base, extra = divmod(samples, workers)
    out, s = [], 0
    for t in range(workers):
        c = base + (1 if t < extra else 0)
        if c:
            out.append((s, s + c))
            s += c
    return out


class CpuInstances:
    """Whole instances of the reference pipeline on the host cores: one
    process per core (as many as CPU_MEM_BUDGET allows), each running a
    contiguous range of the instance's samples — run.sh's process split
    applied to the samples of one instance, so that one instance is one
    step. The pool is started once."""

    def __init__(self, n: int):
        cores = len(os.sched_getaffinity(0))
        self.workers = max(1, min(cores, CPU_MEM_BUDGET // (44 << n), 100))
        self.pool = mp.get_context("spawn").Pool(self.workers)

    def run(self, n: int, m: int, raw, samples: int = 100):
        """(mean P over the samples, wall seconds, kind)."""
        ranges = [(0, samples)] if m == 1 else sample_ranges(samples, self.workers)
        jobs = [(n, m, raw, s0, s1) for s0, s1 in ranges]
        t0 = time.perf_counter()
        res = self.pool.map(_cpu_range_worker, jobs, chunksize=1)
        wall = time.perf_counter() - t0
        kind = "reference" if all(r[2] for r in res) else "port"
        return sum(r[0] for r in res) / samples, wall, kind

    def close(self):
        self.pool.close()
        self.pool.join()


def _step_desc(kind: str) -> str:
    return ("reference Clenshaw_step, MultiQW.cpp:88-173, AVX-512 build" if kind == "reference"
            else "oracle restatement")


def cpu_baseline(n, m, seed, raw=None):
    """One whole seeded n, m instance (all 100 samples; `raw` if given) of the
    reference pipeline, timed on the host cores (about 10 s at n = 20, m = 4
    on 16 cores)."""
    import multistageqw_b200 as M
    cpu = CpuInstances(n)
    try:
        if raw is None:
            raw = M.sk_instances(n, 1, seed)[0]
        cpu.run(n, m, raw, samples=cpu.workers)  # warm-up: one sample per process
        _, wall, kind = cpu.run(n, m, raw)
    finally:
        cpu.close()
    return {
        "value": 1.0 / wall, "unit": "instances/s", "cores": cpu.workers, "kind": kind,
        "sample": (f"one whole n={n}, m={m} instance (100 samples x {m} stages; FP32, "
                   f"{_step_desc(kind)}), its samples split into {cpu.workers} contiguous ranges, "
                   "one process per core"),
        "wall_s": wall,
    }


def cpu_baseline_mixed(ns, ms, raw, samples: int = 4):
    """Bounded sample of a mixed batch: the first `samples` of the 100
    samples of every instance, one (instance, samples) job per process slot,
    one process per core; instances/s = instances x samples/100 / wall."""
    import multistageqw_b200 as M
    cores = len(os.sched_getaffinity(0))
    workers = max(1, min(cores, CPU_MEM_BUDGET // (44 << max(ns))))
    offs = np.cumsum([0] + [M.params_per_instance(n) for n in ns])
    jobs = [(n, m, raw[offs[i]:offs[i + 1]], 0, samples if m > 1 else 100)
            for i, (n, m) in enumerate(zip(ns, ms))]
    # longest first, so that the pool ends together
    jobs.sort(key=lambda j: -(j[4] * j[1] * (1 << j[0])))
    with mp.get_context("spawn").Pool(workers) as pool:
        pool.map(_cpu_range_worker, jobs[:workers], chunksize=1)  # warm-up
        t0 = time.perf_counter()
        res = pool.map(_cpu_range_worker, jobs, chunksize=1)
        wall = time.perf_counter() - t0
    kind = "reference" if all(r[2] for r in res) else "port"
    units = sum((j[4] - j[3]) / 100.0 for j in jobs)
    return {"value": units / wall, "unit": "instances/s", "cores": workers, "kind": kind,
            "sample": (f"the first {samples} of the 100 samples of each of the {len(ns)} "
                       f"instances (m = 1 instances whole; FP32, {_step_desc(kind)}), one "
                       "(instance, samples) job per process, one process per core; "
                       "instances/s = instances x samples/100 / wall"),
            "wall_s": wall}


def _cpu_term_worker(args):
    """Seconds per Clenshaw term (both real halves) of the reference's own
    Clenshaw_step at size n, on seeded vectors."""
    n, reps, seed = args
    sys.path.insert(0, ROOT)
    from oracle import oracle as O
    N = 1 << n
    rng = np.random.default_rng(seed)
    b1 = rng.standard_normal(N).astype(np.float32)
    b2 = rng.standard_normal(N).astype(np.float32)
    hp = rng.standard_normal(N).astype(np.float32)
    psi = rng.standard_normal(N).astype(np.float32)
    use_ref = O.ref_lib() is not None
    step = O.ref_clenshaw_step if use_ref else O.clenshaw_step_f32
    t0 = time.perf_counter()
    for _ in range(reps):
        step(b1, b2, hp, psi, n, 40.0, 1.5, 0.1)  # real half
        step(b1, b2, hp, psi, n, 40.0, 1.5, 0.1)  # imaginary half
    return (time.perf_counter() - t0) / reps, use_ref


def cpu_baseline_per_term(n, terms_per_instance, reps=2):
    """Bounded CPU baseline for large n (a whole n = 28 sample is ~20 min per
    core): every worker times `reps` terms of the reference's step;
    instances/s = workers / (terms per instance x s/term). Workers are capped
    so that their vectors fit CPU_MEM_BUDGET."""
    cores = len(os.sched_getaffinity(0))
    workers = max(1, min(cores, CPU_MEM_BUDGET // (16 << n)))
    with mp.get_context("spawn").Pool(workers) as pool:
        res = pool.map(_cpu_term_worker, [(n, reps, 11 + i) for i in range(workers)])
    sec = max(r[0] for r in res)
    kind = "reference" if all(r[1] for r in res) else "port"
    return {"value": workers / (terms_per_instance * sec), "unit": "instances/s",
            "cores": workers, "kind": kind,
            "sample": (f"{workers} processes x {reps} Clenshaw terms (both halves) at n={n} of the "
                       + ("reference's Clenshaw_step, MultiQW.cpp:88-173, AVX-512 build" if kind == "reference"
                          else "oracle restatement")
                       + f"; {sec:.3f} s/term scaled by {terms_per_instance} terms per instance"),
            "seconds_per_term": sec}


def _cpu_one_sample(args):
    n, m, raw = args
    sys.path.insert(0, ROOT)
    from oracle import oracle as O
    use_ref = O.ref_lib() is not None
    t0 = time.perf_counter()
    r = O.run_problems(n, m, raw, 1, 1, "f32", use_ref_step=use_ref)
    return float(r["p"][0]), time.perf_counter() - t0, use_ref


def cpu_precision_check(raws, n, m):
    """Sample 0 of each instance on the CPU with the reference's own FP32
    Clenshaw_step (partial build) against the GPU's FP32 and FP64 paths."""
    import multistageqw_b200 as M
    ctx = M.Context(0)
    g32 = ctx.run_problems(n, m, raws, samples=1, precision="fp32")["p"]
    g64 = ctx.run_problems(n, m, raws, samples=1, precision="fp64")["p"]
    ctx.close()
    workers = max(1, min(len(raws), CPU_MEM_BUDGET // (44 << n)))
    with mp.get_context("spawn").Pool(workers) as pool:
        res = pool.map(_cpu_one_sample, [(n, m, r) for r in raws])
    cpu = np.array([r[0] for r in res])
    return {"instances": len(raws), "samples": 1, "processes": workers,
            "kind": "reference" if all(r[2] for r in res) else "port",
            "p_cpu": cpu.tolist(), "p_gpu_fp32": g32.tolist(), "p_gpu_fp64": g64.tolist(),
            "max_abs_dP_cpu_vs_gpu_fp64": float(np.abs(cpu - g64).max()),
            "max_abs_dP_gpu_fp32_vs_fp64": float(np.abs(g32 - g64).max()),
            "cpu_seconds_per_sample": float(np.mean([r[1] for r in res]))}


# ---- replicas (one process per GPU, no exchange) ------------------------------

def replica_seed(seed: int, rank: int) -> int:
    """Each rank runs its own seeded batch (independent problems, like the
    reference's run.sh process split)."""
    return seed + 7919 * rank


def max_over_ranks(x: float, world: int, dist=None, device=None) -> float:
    """Max of a per-rank time over all ranks (the job ends when the slowest
    rank ends); identity on one rank."""
    if world <= 1:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# ---- workloads -----------------------------------------------------------------

def make_batch(M, a, rank):
    """(n list, m list, raw concatenated, description) for the workload."""
    seed = replica_seed(a.seed, rank)
    if a.workload == "mixed":
        # The mixed batch (n uniform in {12, 14, 16, 18, 20}, m in {2..5}):
        # its first a.batch instances.
        from multistageqw_b200 import studies
        ns, ms, raw = studies.mixed_batch(a.batch, seed)
        desc = {"workload": "sk_mixed_n12-20_m2-5", "n": "12..20 (even)", "m": "2..5",
                "note": f"{a.batch}-instance seeded batch drawn like the 4096-instance mixed batch"}
        return ns, ms, raw, desc
    if a.workload == "n28":
        raw = M.sk_instances(28, 1, 7)
        desc = {"workload": "sk_n28_m3_seed7", "n": 28, "m": 3,
                "note": f"one instance, {a.samples} of its 100 samples per step; "
                        "instances/s counts samples/100"}
        return [28], [3], raw.ravel(), desc
    if a.workload == "adam_n20_m4":
        raw = adam_instances()[: a.batch]
        desc = {"workload": "adam_sk20n_m4", "n": 20, "m": 4,
                "note": (f"the first {len(raw)} instances of the reference's data/AdamData/SK_20n "
                         "(J ~ N(0, 1/2), h ~ N(0, 1); tests/golden/" + ADAM_FIXTURE + ")")}
        return [20] * len(raw), [4] * len(raw), raw.ravel(), desc
    raw = M.sk_instances(a.n, a.batch, seed)
    desc = {"workload": f"sk_n{a.n}_m{a.m}", "n": a.n, "m": a.m}
    return [a.n] * a.batch, [a.m] * a.batch, raw.ravel(), desc


ADAM_FIXTURE = "adam_sk20n_first16.bin"


def adam_instances():
    """The first 16 instances of the reference's data/AdamData/SK_20n (a
    committed byte copy), [16, 210] float64."""
    import numpy as np
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "tests", "golden", ADAM_FIXTURE)
    return np.fromfile(path, dtype="<f8").reshape(-1, 20 * 21 // 2)


def data_note(a) -> str:
    if a.workload == "adam_n20_m4":
        return "the reference's own AdamData SK_20n instances (committed byte copy)"
    return "synthetic seeded SK instances (J,h ~ N(0,1)); reference datasets not used"


def instance_units(a, count: int) -> float:
    """Instances completed per step (n28 runs a fraction of one instance)."""
    return count * (a.samples / 100.0 if a.workload == "n28" else 1.0)


def reference_arm(a):
    """The reference's own CPU pipeline on the host cores, on this arm's
    workload and metric. n <= 22: every timed step is one whole seeded
    instance (100 samples, split over one process per core; warm-up steps run
    one sample per process). n28: seconds per term of the reference's step,
    scaled to the instance's term count (a whole instance is hours per
    core)."""
    n, m = (28, 3) if a.workload == "n28" else (20, 4) if a.workload == "adam_n20_m4" else (a.n, a.m)
    times, base = [], None
    import multistageqw_b200 as M
    if a.workload == "mixed":
        from multistageqw_b200 import studies
        ns, ms_, raw = studies.mixed_batch(a.batch, replica_seed(a.seed, 0))
        for step in range(a.warmup + a.steps):
            b = cpu_baseline_mixed(ns, ms_, raw)
            if step >= a.warmup:
                times.append(1.0 / b["value"])
            base = b
        config = {"workload": "sk_mixed_n12-20_m2-5", "n": "12..20 (even)", "m": "2..5"}
    elif n > 22:
        for step in range(a.warmup + a.steps):
            # ~1 s per term per core at n = 28: time terms, scale by the
            # instance's term count (3 stages x ~190 terms x 100 samples).
            b = cpu_baseline_per_term(n, 57000, reps=1)
            if step >= a.warmup:
                times.append(1.0 / b["value"])
            base = b
        config = {"workload": f"sk_n{n}_m{m}", "n": n, "m": m, "samples": 100}
    else:
        cpu = CpuInstances(n)
        try:
            adam = adam_instances() if a.workload == "adam_n20_m4" else None
            for step in range(a.warmup + a.steps):
                raw = (adam[step % len(adam)] if adam is not None
                       else M.sk_instances(n, 1, a.seed + 1000 * step)[0])
                if step < a.warmup:
                    cpu.run(n, m, raw, samples=cpu.workers)
                    continue
                _, wall, kind = cpu.run(n, m, raw)
                times.append(wall)
        finally:
            cpu.close()
        base = {"kind": kind, "cores": cpu.workers,
                "sample": (f"every timed step one whole {'AdamData SK_20n' if adam is not None else 'seeded'} "
                           f"n={n}, m={m} instance (100 samples "
                           f"x {m} stages; FP32, {_step_desc(kind)}), its samples split into "
                           f"{cpu.workers} contiguous ranges, one process per core; warm-up steps "
                           "one sample per process")}
        config = {"workload": "adam_sk20n_m4" if adam is not None else f"sk_n{n}_m{m}", "n": n,
                  "m": m, "samples": 100}
    sec = sum(times)
    val = len(times) / sec
    return {
        "metric": METRIC, "value": val, "unit": "instances/s", "n_gpus": a.gpus,
        "steps": a.steps, "warmup": a.warmup, "ms_per_step": 1000.0 * sec / len(times),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": data_note(a),
        "impl": "reference",
        "config": config,
        "cpu_baseline": {k: base[k] for k in ("kind", "cores", "sample")} | {"value": val, "unit": "instances/s"},
        "e2e": {"value": val, "unit": "instances/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def main():
    a = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if a.workload == "n28" and a.samples == 100:
        a.samples = 4

    if a.impl == "reference":
        if rank == 0:
            print(json.dumps(reference_arm(a)), flush=True)
        return

    if a.workload == "mixed_full":
        # The whole 4 096-instance mixed batch in one plan (a study run of
        # a few minutes, not a bench line): one JSON report.
        if rank == 0:
            from multistageqw_b200 import studies
            print(json.dumps(studies.mixed_batch_study(a.batch if a.batch > 2 else 4096)), flush=True)
        return

    if a.workload == "precision":
        if rank == 0:
            from multistageqw_b200 import studies
            # The post-selected draws (screened once on the CPU with the
            # reference's energy arithmetic, tests/golden/make_precision_set.py);
            # the study re-checks every gap on the GPU.
            fx = os.path.join(ROOT, "tests", "golden", "precision_n24_m4.json")
            draws = eloc = None
            if os.path.exists(fx):
                with open(fx) as f:
                    sel = json.load(f)["instances"]
                draws = [s["draw"] for s in sel]
                eloc = [s["e_loc"] for s in sel]
            rep = studies.precision_study(draws=draws, expect_e_loc=eloc)
            raws = rep.pop("raws")
            rep.pop("p_fp32")
            rep.pop("p_fp64")
            if not a.no_cpu:
                rep["cpu_reference"] = cpu_precision_check(raws[:a.cpu_walks], 24, 4)
            print(json.dumps(rep), flush=True)
        return

    import torch
    import torch.distributed as dist

    import multistageqw_b200 as M

    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=600))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    ctx = M.Context(local)
    # A dedicated stream: the library launches (or replays its graph) on the
    # stream it is given, and the CUDA events below are recorded on the same
    # one. (torch's default stream has handle 0, which the ABI reads as "the
    # context's own stream".)
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    ns, ms, raw, desc = make_batch(M, a, rank)
    count = len(ns)
    shape = dict(group=a.group, tile_log=a.tile_log, lanes=a.lanes, threads=a.threads,
                 lane_smem=a.lane_smem, tma=a.tma, cluster=a.cluster)
    plan = M.Plan(ctx, ns, ms, raw, samples=a.samples, precision=a.precision, **shape)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize(dev)

    for _ in range(a.warmup):
        plan.execute(stream.cuda_stream)
    barrier()
    clocks = ClockSampler(gpu_selector(torch, local))
    step_ms, kern_ms = [], []
    term_amps = pass_amps = aux_bytes = 0.0
    launches = term_launches = terms = 0
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
        pass_amps += st["pass_amps"]
        aux_bytes += st["aux_bytes"]
        launches += st["launches"]
        term_launches += st["term_launches"]
        terms = st["terms"]
    barrier()
    clk = clocks.stop()
    total_ms = max_over_ranks(sum(step_ms), world, dist, dev)
    value = world * instance_units(a, count) * a.steps / (total_ms / 1000.0)

    # End to end through the public API from pinned host buffers.
    raw_pinned = torch.from_numpy(np.ascontiguousarray(raw)).pin_memory().numpy()
    e2e_ms = []
    e2e_parts = {"create_ms": 0.0, "execute_call_ms": 0.0, "results_ms": 0.0}
    h2d = d2h = 0.0
    for it in range(1 + max(2, min(a.steps, 3))):  # the first one is an untimed warm-up
        flush.zero_()
        barrier()
        t0 = time.perf_counter()
        p2 = M.Plan(ctx, ns, ms, raw_pinned, samples=a.samples, precision=a.precision,
                    graph=0, **shape)
        t1 = time.perf_counter()
        p2.execute()
        t2 = time.perf_counter()
        r = p2.results()
        torch.cuda.synchronize(dev)
        t3 = time.perf_counter()
        st2 = p2.stats()
        if it == 0:
            p2.close()
            continue
        e2e_ms.append((t3 - t0) * 1000.0)
        e2e_parts["create_ms"] += (t1 - t0) * 1000.0
        e2e_parts["execute_call_ms"] += (t2 - t1) * 1000.0
        e2e_parts["results_ms"] += (t3 - t2) * 1000.0
        h2d, d2h = st2["h2d_bytes"], st2["d2h_bytes"]
        p2.close()
    e2e_parts = {k: v / len(e2e_ms) for k, v in e2e_parts.items()}
    e2e_total = max_over_ranks(sum(e2e_ms), world, dist, dev)
    e2e_val = world * instance_units(a, count) * len(e2e_ms) / (e2e_total / 1000.0)

    # |dP| of every timed FP32 result against the FP64 path (same instances,
    # same samples), and the state-vector error of one walk (instance 0,
    # sample 0) after its last stage, FP32 against FP64.
    check = None
    res = plan.results()
    if not a.no_check and a.precision != "fp64":
        r64p = M.Plan(ctx, ns, ms, raw, samples=a.samples, precision="fp64", graph=0)
        r64p.execute()
        r64 = r64p.results()
        r64p.close()
        dP = np.abs(res["p"] - r64["p"])
        check = {"max_abs_dP_vs_fp64": float(dP.max()), "mean_abs_dP_vs_fp64": float(dP.mean()),
                 "instances_checked": len(ns), "tolerance": 1e-5,
                 "e_loc_equal": bool(np.array_equal(res["e_loc"], r64["e_loc"])),
                 "p_fp32": [float(x) for x in res["p"][:8]],
                 "p_fp64": [float(x) for x in r64["p"][:8]]}
        if max(ns) <= 24:
            from multistageqw_b200 import studies
            per0 = M.params_per_instance(ns[0])
            s32, _, eloc = studies.stage_states(ctx, ns[0], ms[0], raw[:per0], 0, "fp32")
            s64, _, _ = studies.stage_states(ctx, ns[0], ms[0], raw[:per0], 0, "fp64")
            check["state_rel_l2_vs_fp64"] = float(np.linalg.norm(s32[-1] - s64[-1]) /
                                                  np.linalg.norm(s64[-1]))
            check["state_rel_l2_per_stage"] = [float(np.linalg.norm(x - y) / np.linalg.norm(y))
                                               for x, y in zip(s32, s64)]
            check["state_walk"] = "instance 0, sample 0, stage by stage through mqw_clenshaw"

    pk, pk_kind = peaks()
    tiers = ctx.measure_peaks() if rank == 0 else None
    kms = sum(kern_ms)
    # The dominant kernel, pass_kernel (one fused Clenshaw pass), timed alone:
    # CUDA events on the launching stream around a pass-only replay in the
    # plan's own autotuned shape (walks per launch, concurrent lanes) for the
    # workload's largest n. Its algorithmic bytes per launch are 36 B per
    # term·amp (FP32; 72 B in FP64) x 2^n x walks per launch.
    n_dom = int(max(ns))
    # When the shared-basis chains carry more bytes than the walks' own
    # passes (FP32 with the product bases: at n = 20, m = 4 no walk runs a
    # recurrence), the dominant kernel is the real chain pass instead:
    # 16 B per amplitude algorithmic (read b_{r+1}, b_{r+2}, D; write b_r),
    # timed alone the same way (mqw_chain_pass_timing).
    chain_dom = a.precision == "fp32" and BYTES_PER_TERM_AMP["fp32"] * pass_amps < aux_bytes
    if chain_dom:
        pt = ctx.chain_pass_timing(n_dom, reps=64)
        per_amp, vec_bytes, kname = CHAIN_BYTES_PER_AMP, 4, "real_pass_kernel"
    else:
        pt = ctx.pass_timing(n_dom, a.precision if a.precision != "fp32c" else "fp32", reps=64)
        per_amp = BYTES_PER_TERM_AMP[a.precision]
        vec_bytes, kname = (8 if a.precision != "fp64" else 16), "pass_kernel"
    bytes_per_launch = per_amp * float(1 << n_dom) * pt["walks_per_launch"]
    achieved = bytes_per_launch / (pt["us_per_launch"] * 1e-6) / 1e9
    # Bound tier: the memory tier that holds the concurrent walks' (chains')
    # working set (3 vectors per walk or chain in flight, and the instance's
    # 4 B diagonal, which they share): L2 (126 MB; the library's own L2 copy
    # probe is the denominator) when it fits in 96 MB, else HBM
    # (MEASURED_PEAKS.json).
    ws = (3 * vec_bytes * pt["walks_per_launch"] * pt["lanes"] + 4) * float(1 << n_dom)
    l2_resident = ws <= 96e6 and tiers is not None
    if l2_resident:
        bound, peak, peak_src = "l2", tiers["l2_copy_gbs"], "l2_copy_gbs of the library's own probe"
    else:
        bound, peak, peak_src = "hbm", pk["hbm_gbs"], f"hbm_gbs of {pk_kind}"
    dram = (CHAIN_DRAM_BYTES_PER_AMP if chain_dom else DRAM_BYTES_PER_TERM_AMP).get(desc["workload"])
    # Propagation phase as a whole (every pass plus the shared-basis kernels'
    # reads and writes, over the plan's device time): context for the
    # kernel figure above.
    moved = BYTES_PER_TERM_AMP[a.precision] * pass_amps + aux_bytes
    phase_gbs = moved / (kms / 1000.0) / 1e9 if kms > 0 else None
    roofline = {
        "bound": bound, "achieved": achieved, "peak": peak, "unit": "GB/s",
        "frac": achieved / peak, "traffic": dram * float(1 << n_dom) * pt["walks_per_launch"] if dram else None,
        "peak_source": peak_src,
        "kernel": (f"{kname} at n={n_dom}: frac = bytes_per_launch / avg_launch_us / peak; "
                   "avg_launch_us from CUDA events around a pass-only replay in the plan's tuned "
                   f"shape ({pt['walks_per_launch']} walk(s) or chain(s) per launch, "
                   f"{pt['lanes']} lane(s) in flight, so it is the launch-to-launch time); "
                   f"bytes_per_launch = {per_amp} B per amplitude algorithmic; traffic = "
                   "cold-cache DRAM bytes per launch from ncu"),
        "bytes_per_launch": bytes_per_launch,
        "avg_launch_us": pt["us_per_launch"],
        "walks_per_launch": pt["walks_per_launch"], "lanes": pt["lanes"],
        "working_set_bytes": ws,
        "phase": {"achieved_gbs": phase_gbs, "device_ms_per_step": kms / max(1, a.steps),
                  "algorithmic_bytes_per_step": moved / max(1, a.steps),
                  "note": "whole propagation phase: executed passes at 36 B per term·amp plus "
                          "the shared-basis kernels' reads and writes, over the phase's device time"},
    }
    # FP32 arithmetic of the pass kernel: (2n + 8) FLOP per term·amp (the
    # diagonal product, the n partner sums and the Clenshaw update, complex)
    # per launch over its launch-to-launch time, against the SIMT FP32 peak
    # at the maximum SM clock (the kernel is memory-bound; this is the
    # compute roof it stays far below).
    if a.precision != "fp64" and not chain_dom:
        sms = torch.cuda.get_device_properties(dev).multi_processor_count
        mhz = float((clk or {}).get("sm_max_mhz") or 1965.0)
        peak_tf = sms * 128 * 2 * mhz * 1e6 / 1e12
        ex_tf = (2 * n_dom + 8) * float(1 << n_dom) * pt["walks_per_launch"] / \
            (pt["us_per_launch"] * 1e-6) / 1e12
        roofline["fp32_flops"] = {"per_term_amp": 2 * n_dom + 8, "achieved_tflops": ex_tf,
                                  "peak_tflops": peak_tf, "frac": ex_tf / peak_tf}
    # The chain pass's binding resource, the SM's L1 data pipe: its
    # wavefronts per launch (ncu) over the launch-to-launch time's cycles on
    # all SMs (one wavefront per cycle per SM, at the median sampled clock).
    wf = CHAIN_L1_WAVEFRONTS_PER_AMP.get(n_dom) if chain_dom and pt["walks_per_launch"] == 1 else None
    if wf:
        sms = torch.cuda.get_device_properties(dev).multi_processor_count
        mhz = float((clk or {}).get("sm_mhz") or (clk or {}).get("sm_max_mhz") or 1965.0)
        per_launch = wf * float(1 << n_dom)
        roofline["l1_pipe"] = {
            "wavefronts_per_launch": per_launch, "sm_mhz": mhz, "sms": sms,
            "frac": per_launch / (pt["us_per_launch"] * 1e-6 * mhz * 1e6 * sms),
            "note": "L1 data-pipe (LSU: shared memory, shuffles, global) wavefronts of one "
                    "launch from ncu over the launch-to-launch cycles of all SMs at one "
                    "wavefront per cycle per SM"}
    if tiers:
        roofline["tiers_gbs"] = {k: round(v, 1) for k, v in tiers.items()}
        roofline["frac_of_hbm"] = achieved / pk["hbm_gbs"]

    if rank == 0:
        cpu = None
        if world == 1 and not a.no_cpu:
            try:
                if a.workload == "n28":
                    cpu = cpu_baseline_per_term(28, int(terms * 100.0 / a.samples))
                elif a.workload == "mixed":
                    cpu = cpu_baseline_mixed(ns, ms, raw)
                elif a.workload == "adam_n20_m4":
                    cpu = cpu_baseline(20, 4, 0, raw=adam_instances()[0])
                else:
                    cpu = cpu_baseline(a.n, a.m, 4242)
            except Exception as ex:  # the baseline is reported, not required
                cpu = {"value": None, "error": str(ex)}
        config = dict(desc)
        if not (a.group or a.tile_log or a.lanes or a.threads or a.lane_smem or a.tma
                or a.cluster):
            config["grid_shape"] = ctx.grid_shape(max(ns), a.precision)
        config["reference_term_amps_per_step"] = term_amps / a.steps
        config["pass_term_amps_per_step"] = pass_amps / a.steps
        config["shared_basis_bytes_per_step"] = aux_bytes / a.steps
        config.update({"instances_per_step": count * world, "samples": a.samples,
                       "precision": a.precision, "group": a.group or "autotuned",
                       "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                       "l2": "flushed between timed steps (256 MB write)",
                       "graph": "CUDA graph replay of the whole device pipeline",
                       "stage2_product_basis": {"0": "off", "1": "forced"}.get(
                           os.environ.get("MQW_STAGE2_BASIS", ""),
                           "auto (when 2 x stage-1 basis size <= walks per instance)")})
        line = {
            "metric": METRIC, "value": value, "unit": "instances/s", "n_gpus": world,
            "steps": a.steps, "warmup": a.warmup, "ms_per_step": total_ms / a.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if a.precision == "fp64" else "f32",
            "data": data_note(a),
            "config": config,
            "e2e": {"value": e2e_val, "unit": "instances/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "per_step": e2e_parts},
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
