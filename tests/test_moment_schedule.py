"""The higher-moment stage heuristic (skewness and kurtosis of H_P through
the Cornish-Fisher expansion): its pieces on the CPU, its equal-cost
application and its evaluation against the paper heuristic on the GPU."""
import math

import numpy as np
import pytest


def test_central_moments_of_a_known_sample(mqw):
    from multistageqw_b200 import moment_schedule as MS
    rng = np.random.default_rng(3)
    x = rng.gamma(4.0, 1.0, 200000)  # skewness 2/sqrt(4) = 1, excess kurtosis 6/4 = 1.5
    raw = [float(np.mean(x ** k)) for k in range(1, 5)]
    var, g1, g2 = MS.central_moments(raw)
    assert var == pytest.approx(np.var(x), rel=1e-9)
    assert g1 == pytest.approx(1.0, abs=0.05)
    assert g2 == pytest.approx(1.5, abs=0.2)


def test_cornish_fisher_depth(mqw):
    from multistageqw_b200 import moment_schedule as MS
    # Gaussian: the depth is the normal depth itself.
    assert MS.cornish_fisher_depth(3.7, 0.0, 0.0) == pytest.approx(3.7, abs=1e-15)
    # A left-skewed (negative g1) distribution has a longer lower tail.
    assert MS.cornish_fisher_depth(3.7, -0.2, 0.0) > 3.7
    # Heavier tails (positive excess kurtosis) reach further.
    assert MS.cornish_fisher_depth(3.7, 0.0, 0.3) > 3.7


def test_heuristic_depth_matches_the_schedule(mqw, orc):
    """a of MultiQW.cpp:367-370, recomputed in double, reproduces the gammas
    of the (bit-exact) heuristic schedule to float precision."""
    from multistageqw_b200 import moment_schedule as MS
    n, m = 14, 3
    raw = orc.sk_instances(n, 1, 21)[0]
    g, _, _, _ = orc.schedule(n, m, raw)
    npair = n * (n - 1) // 2
    J = raw[:npair].astype(np.float32).astype(np.float64)
    h = raw[npair:].astype(np.float32).astype(np.float64)
    hp2 = float(np.sum(J * J) + np.sum(h * h))
    a = MS.heuristic_depth(n)
    for i in range(m):
        want = a * math.sqrt(hp2) / math.tan(math.pi * (i + 1) / (2 * m + 2)) / n
        assert float(g[i]) == pytest.approx(want, rel=3e-6)


@pytest.mark.gpu
def test_moment_heuristic_runs_at_equal_cost(ctx, mqw):
    """The higher-moment heuristic on 48 fresh n = 14, m = 4 instances:
    finite gamma factors, the same Chebyshev work as the paper heuristic
    (within 1%), valid probabilities. Whether it gains is reported by
    `python -m multistageqw_b200.moment_schedule`, not asserted."""
    from multistageqw_b200 import moment_schedule as MS
    r = MS.evaluate(ctx, 14, 4, 48, 9914, samples=20)
    assert abs(r["terms_moments"] / r["terms_heuristic"] - 1.0) < 0.01
    assert 0.0 < r["mean_p_moments"] <= 1.0 and 0.0 < r["mean_p_heuristic"] <= 1.0
    lo, hi = r["gamma_factor_range"]
    assert 0.5 < lo <= hi < 2.0
