"""Higher-moment stage heuristic: the paper's hopping rates corrected by the
skewness and kurtosis of the energy diagonal.

The paper heuristic (MultiQW.cpp:365-375, 392) sets

    gamma_i = a sqrt(HP2) / tan(pi (i + 1) / (2m + 2)) / n,

where sqrt(HP2) is the standard deviation of the Ising energies over the 2^n
basis states and a = (1 - g_E) Q^-1(1/N) + g_E Q^-1(1/(eN)) (g_E the
Euler–Mascheroni constant, Q^-1 the upper-tail normal quantile) is the
expected maximum of N = 2^n standard normals: a sqrt(HP2) estimates how far
the ground energy lies below the mean energy as if the energies were
Gaussian. The reference notes (MultiQW.cpp:379-383, commented out) that the
skewness and kurtosis of H_P could refine that estimate. Here they do: with
the central moments of H_P computed on the GPU in FP64 (mqw_diag_moments),
the lower-tail quantile at the same depth is taken from the Cornish–Fisher
expansion (Cornish & Fisher 1938; the standard four-moment form)

    w(z) = z + (z^2 - 1) g1/6 + (z^3 - 3z) g2/24 - (2z^3 - 5z) g1^2/36

at z = -a (g1 the skewness, g2 the excess kurtosis), so the ground energy is
estimated -w(-a) standard deviations below the mean instead of a. Every
stage's gamma is scaled by -w(-a)/a (and by the ratio of the GPU's standard
deviation to sqrt(HP2), which is 1 up to float rounding); the times are then
rescaled by one common factor so that the Chebyshev work, sum_i
onenorm_i t_i, equals the paper heuristic's (the same equal-cost rule as the
learned schedule). The heuristic's own schedule is the fallback whenever the
correction is not finite.

No counterpart in the reference beyond the comment; `evaluate` compares it
with the paper heuristic at equal simulated cost, the simulator's P as the
judge.
"""
from __future__ import annotations

import math

import numpy as np

from . import Context, inv_norm_upper, schedule, sk_instances
from .learned import equal_cost_scale, run_with_scale

EULER_GAMMA = 0.5772156649015329


def heuristic_depth(n: int) -> float:
    """The paper heuristic's a (MultiQW.cpp:367-370), in double."""
    N = float(1 << n)
    b = float(inv_norm_upper(1.0 / N))
    return (1.0 - EULER_GAMMA) * b + EULER_GAMMA * float(inv_norm_upper(1.0 / (math.e * N)))


def cornish_fisher_depth(a: float, g1: float, g2: float) -> float:
    """-w(-a): the lower-tail depth, in standard deviations, of a distribution
    with skewness g1 and excess kurtosis g2 at the normal depth a."""
    z = -a
    w = z + (z * z - 1.0) * g1 / 6.0 + (z ** 3 - 3.0 * z) * g2 / 24.0 - \
        (2.0 * z ** 3 - 5.0 * z) * g1 * g1 / 36.0
    return -w


def central_moments(raw_moments) -> tuple[float, float, float]:
    """(variance, skewness, excess kurtosis) from mean(x^k), k = 1..4."""
    m1, m2, m3, m4 = (float(x) for x in raw_moments)
    var = m2 - m1 * m1
    c3 = m3 - 3.0 * m1 * m2 + 2.0 * m1 ** 3
    c4 = m4 - 4.0 * m1 * m3 + 6.0 * m1 * m1 * m2 - 3.0 * m1 ** 4
    return var, c3 / var ** 1.5, c4 / (var * var) - 3.0


def moment_stage_scale(ctx: Context, n: int, m: int, raws: np.ndarray) -> tuple[np.ndarray, list]:
    """[count, m, 2] (gamma, t) multipliers of the higher-moment heuristic at
    equal cost, and per instance (skewness, excess kurtosis, gamma factor)."""
    raws = np.asarray(raws, np.float64).reshape(len(raws), -1)
    out = np.ones((len(raws), m, 2), np.float32)
    stats = []
    a = heuristic_depth(n)
    npair = n * (n - 1) // 2
    for k, r in enumerate(raws):
        var, g1, g2 = central_moments(ctx.diag_moments(n, r))
        _, _, info = ctx.build_diag(n, r)
        g, st, _, _ = schedule(n, m, r)
        # sqrt(HP2) of MultiQW.cpp:375 (J symmetrised and halved, as read)
        J = r[:npair].astype(np.float32).astype(np.float64) / 2.0
        h = r[npair:].astype(np.float32).astype(np.float64)
        hp2 = 4.0 * float(np.sum(J * J)) + float(np.sum(h * h))
        fac = cornish_fisher_depth(a, g1, g2) / a * math.sqrt(var / hp2)
        stats.append((g1, g2, fac))
        if not (math.isfinite(fac) and fac > 0):
            continue
        dlg = np.full(m, math.log(fac))
        sc = equal_cost_scale(n, g, st, float(info.e_abs), dlg, np.zeros(m))
        if np.all(np.isfinite(sc)) and np.all(sc > 0):
            out[k] = sc
    return out, stats


def evaluate(ctx: Context, n: int, m: int, count: int, seed: int, samples: int = 100) -> dict:
    """Mean P of the paper heuristic and of the higher-moment heuristic (equal
    cost) on `count` fresh seeded SK instances (J, h ~ N(0, 1))."""
    raws = sk_instances(n, count, seed)
    p_h, terms_h = run_with_scale(ctx, n, m, raws, None, samples)
    scale, stats = moment_stage_scale(ctx, n, m, raws)
    p_m, terms_m = run_with_scale(ctx, n, m, raws, scale, samples)
    g1 = np.array([s[0] for s in stats])
    g2 = np.array([s[1] for s in stats])
    fac = np.array([s[2] for s in stats])
    return {"n": n, "m": m, "instances": count, "samples": samples,
            "mean_p_heuristic": float(p_h.mean()), "mean_p_moments": float(p_m.mean()),
            "ratio": float(p_m.mean() / p_h.mean()),
            "frac_instances_improved": float(np.mean(p_m > p_h)),
            "terms_heuristic": int(terms_h), "terms_moments": int(terms_m),
            "skewness_mean": float(g1.mean()), "excess_kurtosis_mean": float(g2.mean()),
            "gamma_factor_mean": float(fac.mean()), "gamma_factor_range": [float(fac.min()),
                                                                           float(fac.max())]}


def main(argv=None) -> None:
    import argparse
    import json
    ap = argparse.ArgumentParser(description="evaluate the higher-moment stage heuristic")
    ap.add_argument("--n", default="14,18,20")
    ap.add_argument("--m", type=int, default=4)
    ap.add_argument("--count", type=int, default=256)
    ap.add_argument("--samples", type=int, default=100)
    a = ap.parse_args(argv)
    ctx = Context(0)
    rep = [evaluate(ctx, int(n), a.m, a.count, 9000 + int(n), a.samples) for n in a.n.split(",")]
    ctx.close()
    print(json.dumps(rep), flush=True)


if __name__ == "__main__":
    main()
