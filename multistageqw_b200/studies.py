"""Precision study on near-degenerate instances (n = 24, m = 4).

Seeded SK instances (J, h ~ N(0,1)) are drawn until `count` of them have a
gap E_(1) - E_(0) < gap_max between their two lowest energies (the energies
of the reference's arithmetic, the ones that define E_loc). On those:

* the whole path in FP32 and in FP64 on the GPU (`samples` samples each):
  per-instance |dP|;
* for `state_walks` walks, the state after every stage in FP32 and FP64
  (stage by stage through mqw_clenshaw): relative L2 error per stage;
* the Chebyshev degree per stage (mean over samples);
* instances whose gap is below 1e-4 are flagged (there the reference's
  float-increment energies could order the two lowest states differently
  from exact arithmetic).
"""
from __future__ import annotations

import time

import numpy as np

from . import Context, cheb_coeffs_host, schedule, sk_instances


def screen(ctx: Context, n: int, count: int, seed: int, gap_max: float, max_draws: int):
    kept = []
    draws = 0
    t0 = time.time()
    while len(kept) < count and draws < max_draws:
        raw = sk_instances(n, 1, seed * 1_000_003 + draws)[0]
        _, E, info = ctx.build_diag(n, raw, energies=True)
        two = np.partition(E, 1)[:2]
        gap = float(two[1] - two[0])
        if gap < gap_max:
            kept.append({"raw": raw, "gap": gap, "e_loc": int(info.e_loc), "e_abs": float(info.e_abs),
                         "draw": draws})
        draws += 1
    return kept, draws, time.time() - t0


def stage_states(ctx: Context, n: int, m: int, raw, sample: int, precision: str):
    """States after each stage of one walk (normalised), via mqw_clenshaw."""
    hp, _, info = ctx.build_diag(n, raw)
    g, _, times, _ = schedule(n, m, raw)
    N = 1 << n
    cdt = np.complex64 if precision == "fp32" else np.complex128
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


def precision_study(n: int = 24, m: int = 4, count: int = 32, seed: int = 24,
                    gap_max: float = 1e-2, samples: int = 4, max_draws: int = 4000,
                    state_walks: int = 2) -> dict:
    ctx = Context(0)
    kept, draws, t_screen = screen(ctx, n, count, seed, gap_max, max_draws)
    raws = np.stack([k["raw"] for k in kept])
    t0 = time.time()
    r32 = ctx.run_problems(n, m, raws, samples=samples, precision="fp32")
    t32 = time.time() - t0
    t0 = time.time()
    r64 = ctx.run_problems(n, m, raws, samples=samples, precision="fp64")
    t64 = time.time() - t0
    dP = np.abs(r32["p"] - r64["p"])
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
        s64, _, _ = stage_states(ctx, n, m, kept[w]["raw"], 0, "fp64")
        state_err.append({
            "instance": w,
            "rel_l2_per_stage": [float(np.linalg.norm(a - b) / np.linalg.norm(b)) for a, b in zip(s32, s64)],
            "dP_sample0": float(abs(abs(s32[-1][eloc]) ** 2 - abs(s64[-1][eloc]) ** 2)),
        })
    ctx.close()
    return {
        "metric": "precision study: FP32 vs FP64 on near-degenerate SK instances",
        "n": n, "m": m, "instances": len(kept), "draws_screened": draws, "gap_max": gap_max,
        "screen_seconds": t_screen, "samples": samples,
        "gaps": [k["gap"] for k in kept],
        "gaps_below_1e-4": int(sum(k["gap"] < 1e-4 for k in kept)),
        "max_abs_dP": float(dP.max()), "mean_abs_dP": float(dP.mean()),
        "p_fp32_mean": float(r32["p"].mean()), "p_fp64_mean": float(r64["p"].mean()),
        "e_loc_fp32_equals_fp64": bool(np.array_equal(r32["e_loc"], r64["e_loc"])),
        "degree_per_stage_mean": deg.mean(axis=0).tolist(),
        "seconds_fp32": t32, "seconds_fp64": t64,
        "state_error": state_err,
        "raws": raws,  # for the caller's CPU comparison; dropped before printing
        "p_fp32": r32["p"], "p_fp64": r64["p"],
    }
