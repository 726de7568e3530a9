"""Precision study on near-degenerate instances (n = 24, m = 4).

The instances are seeded SK draws (J, h ~ N(0,1)) whose two lowest energies
E_(1) - E_(0) differ by less than `gap_max` (energies in the reference's
arithmetic, the ones that define E_loc). The kept draws either come as a
list (a precomputed screen; every gap is re-checked here on the GPU) or are
screened here on the GPU. On them:

* the whole path in FP32, in FP32 with compensated partner sums and in FP64
  on the GPU (`samples` samples each): per-instance |dP| and the
  ground-state index of the paths;
* for `state_walks` walks, the state after every stage in FP32, compensated
  FP32 and FP64 (stage by stage through mqw_clenshaw): relative L2 error per
  stage;
* the Chebyshev degree per stage (mean over samples);
* instances whose gap is below 1e-4 are flagged (there the reference's
  float-increment energies could order the two lowest states differently
  from exact arithmetic).
"""
from __future__ import annotations

import time

import numpy as np

from . import Context, cheb_coeffs_host, schedule

DRAW_SEED = 24 * 1_000_003  # draw d is default_rng(DRAW_SEED + d)


def draw_raw(n: int, d: int) -> np.ndarray:
    """Draw d of the study: n(n+1)/2 standard normals (J pairs, then h)."""
    return np.random.default_rng(DRAW_SEED + d).standard_normal(n * (n + 1) // 2)


def two_lowest_gap(ctx: Context, n: int, raw):
    """(E_(1) - E_(0), E_loc, E_abs) from the GPU diagonal."""
    _, E, info = ctx.build_diag(n, raw, energies=True)
    i = int(E.argmin())
    e0 = E[i]
    E[i] = np.inf
    return float(E.min() - e0), int(info.e_loc), float(info.e_abs)


def screen(ctx: Context, n: int, count: int, gap_max: float, max_draws: int, draws=None):
    kept = []
    t0 = time.time()
    cand = range(max_draws) if draws is None else draws
    seen = 0
    for d in cand:
        if len(kept) >= count:
            break
        raw = draw_raw(n, int(d))
        gap, e_loc, e_abs = two_lowest_gap(ctx, n, raw)
        seen += 1
        if gap < gap_max:
            kept.append({"raw": raw, "gap": gap, "e_loc": e_loc, "e_abs": e_abs, "draw": int(d)})
        elif draws is not None:
            raise ValueError(f"draw {d}: gap {gap} is not below {gap_max}")
    return kept, seen, time.time() - t0


def stage_states(ctx: Context, n: int, m: int, raw, sample: int, precision: str):
    """States after each stage of one walk (normalised), via mqw_clenshaw."""
    hp, _, info = ctx.build_diag(n, raw)
    g, _, times, _ = schedule(n, m, raw)
    N = 1 << n
    cdt = np.complex128 if precision == "fp64" else np.complex64
    psi = np.full(N, np.float32(1.0 / np.sqrt(N)), dtype=cdt)
    out, degrees = [], []
    for i in range(m):
        onenorm = np.float32(np.float32(info.e_abs) + np.float32(g[i]) * np.float32(n))
        s = float(np.float32(onenorm * times[i, sample]))
        c, K = cheb_coeffs_host(s)
        degrees.append(int(K[0]))
        psi = ctx.clenshaw(n, c[0], hp, float(g[i]), float(onenorm), psi, precision)
        psi = psi / np.linalg.norm(psi.astype(np.complex128))
        out.append(psi.astype(np.complex128))
    return out, degrees, int(info.e_loc)


def precision_study(n: int = 24, m: int = 4, count: int = 32, gap_max: float = 1e-2,
                    samples: int = 4, max_draws: int = 20000, state_walks: int = 2,
                    draws=None, expect_e_loc=None) -> dict:
    """Runs the study; `draws` (optional) lists the kept draw indices of a
    precomputed screen and `expect_e_loc` their ground-state indices."""
    ctx = Context(0)
    kept, seen, t_screen = screen(ctx, n, count, gap_max, max_draws, draws)
    raws = np.stack([k["raw"] for k in kept])
    t0 = time.time()
    r32 = ctx.run_problems(n, m, raws, samples=samples, precision="fp32")
    t32 = time.time() - t0
    t0 = time.time()
    r32c = ctx.run_problems(n, m, raws, samples=samples, precision="fp32c")
    t32c = time.time() - t0
    t0 = time.time()
    r64 = ctx.run_problems(n, m, raws, samples=samples, precision="fp64")
    t64 = time.time() - t0
    dP = np.abs(r32["p"] - r64["p"])
    dPc = np.abs(r32c["p"] - r64["p"])
    # Degrees per stage (the same rule the GPU applies), mean over samples.
    deg = np.zeros((len(kept), m))
    for k, inst in enumerate(kept):
        g, _, times, _ = schedule(n, m, inst["raw"])
        for i in range(m):
            onenorm = np.float32(np.float32(inst["e_abs"]) + np.float32(g[i]) * np.float32(n))
            s = (np.float32(onenorm) * times[i, :samples].astype(np.float32)).astype(np.float64)
            _, K = cheb_coeffs_host(s)
            deg[k, i] = K.mean()
    state_err = []
    for w in range(min(state_walks, len(kept))):
        s32, _, eloc = stage_states(ctx, n, m, kept[w]["raw"], 0, "fp32")
        s32c, _, _ = stage_states(ctx, n, m, kept[w]["raw"], 0, "fp32c")
        s64, _, _ = stage_states(ctx, n, m, kept[w]["raw"], 0, "fp64")
        state_err.append({
            "instance": w,
            "rel_l2_per_stage": [float(np.linalg.norm(a - b) / np.linalg.norm(b)) for a, b in zip(s32, s64)],
            "rel_l2_per_stage_compensated": [float(np.linalg.norm(a - b) / np.linalg.norm(b))
                                             for a, b in zip(s32c, s64)],
            "dP_sample0": float(abs(abs(s32[-1][eloc]) ** 2 - abs(s64[-1][eloc]) ** 2)),
        })
    ctx.close()
    e_loc = [k["e_loc"] for k in kept]
    rep = {
        "metric": "precision study: FP32 vs FP64 on near-degenerate SK instances",
        "n": n, "m": m, "instances": len(kept), "draws_screened": seen, "gap_max": gap_max,
        "screen": "precomputed list, gaps re-checked on the GPU" if draws is not None else "GPU screen",
        "screen_seconds": t_screen, "samples": samples,
        "gaps": [k["gap"] for k in kept],
        "gaps_below_1e-4": int(sum(k["gap"] < 1e-4 for k in kept)),
        "max_abs_dP": float(dP.max()), "mean_abs_dP": float(dP.mean()),
        "max_abs_dP_compensated": float(dPc.max()), "mean_abs_dP_compensated": float(dPc.mean()),
        "seconds_fp32_compensated": t32c,
        "p_fp32_mean": float(r32["p"].mean()), "p_fp64_mean": float(r64["p"].mean()),
        "e_loc_fp32_equals_fp64": bool(np.array_equal(r32["e_loc"], r64["e_loc"])),
        "degree_per_stage_mean": deg.mean(axis=0).tolist(),
        "seconds_fp32": t32, "seconds_fp64": t64,
        "state_error": state_err,
        "raws": raws,  # for the caller's CPU comparison; dropped before printing
        "p_fp32": r32["p"], "p_fp64": r64["p"],
    }
    if expect_e_loc is not None:
        rep["e_loc_equals_screen"] = bool(list(expect_e_loc)[:len(e_loc)] == e_loc)
    return rep


def mixed_batch(count: int = 4096, seed: int = 0):
    """The mixed batch: `count` seeded SK instances (J, h ~ N(0,1)) with n
    uniform in {12, 14, 16, 18, 20} and m uniform in {2, 3, 4, 5}. Returns
    (n list, m list, raw values back to back)."""
    from . import sk_instances
    rng = np.random.default_rng(seed)
    ns = rng.choice([12, 14, 16, 18, 20], count).tolist()
    ms = rng.integers(2, 6, count).tolist()
    raws = [sk_instances(n, 1, int(rng.integers(1 << 31)))[0] for n in ns]
    return ns, ms, np.concatenate(raws)


def mixed_batch_study(count: int = 4096, seed: int = 0, fp64_subset: int = 128) -> dict:
    """The whole mixed batch as one plan in FP32 (timed after a warm-up plan
    that tunes every n), and its first `fp64_subset` instances again in FP64
    for |dP| per instance."""
    from . import Plan, params_per_instance
    ns, ms, raw = mixed_batch(count, seed)
    ctx = Context(0)
    # Tune each n once (the autotuner's timing is not part of the batch).
    warm_idx = [ns.index(n) for n in sorted(set(ns))]
    offs = np.cumsum([0] + [params_per_instance(n) for n in ns])
    warm_raw = np.concatenate([raw[offs[i]:offs[i + 1]] for i in warm_idx])
    wp = Plan(ctx, [ns[i] for i in warm_idx], [ms[i] for i in warm_idx], warm_raw, samples=2, graph=0)
    wp.execute()
    wp.results()
    wp.close()
    t0 = time.time()
    plan = Plan(ctx, ns, ms, raw, graph=0)
    t_create = time.time() - t0
    t1 = time.time()
    plan.execute()
    r32 = plan.results()
    t_exec = time.time() - t1
    st = plan.stats()
    plan.close()
    k = min(fp64_subset, count)
    sub = raw[:offs[k]]
    p64 = Plan(ctx, ns[:k], ms[:k], sub, precision="fp64", graph=0)
    t2 = time.time()
    p64.execute()
    r64 = p64.results()
    t_64 = time.time() - t2
    p64.close()
    ctx.close()
    dP = np.abs(r32["p"][:k] - r64["p"])
    by_n = {}
    for n in sorted(set(ns)):
        idx = [i for i in range(count) if ns[i] == n]
        by_n[str(n)] = {"instances": len(idx), "mean_p": float(np.mean(r32["p"][idx]))}
    return {
        "metric": "mixed batch: instances/s over the whole batch (FP32), |dP| vs FP64",
        "instances": count, "seed": seed, "n": "12..20 (even)", "m": "2..5",
        "seconds_create": t_create, "seconds_execute_and_read": t_exec,
        "instances_per_s": count / t_exec,
        "device_ms_propagation": st["kernel_ms"], "launches": st["launches"],
        "term_amps": st["term_amps"], "pass_amps": st["pass_amps"],
        "fp64_subset": k, "seconds_fp64_subset": t_64,
        "max_abs_dP": float(dP.max()), "mean_abs_dP": float(dP.mean()),
        "by_n": by_n,
    }
