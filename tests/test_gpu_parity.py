"""GPU parity tests: every device piece and the whole path, called through
the C ABI, against the oracle on the same seeded inputs.

Bars:
  * diagonal (energies, H_P, E_loc, E_abs): bit-exact;
  * Chebyshev degrees and float coefficients: bit-exact;
  * FP64 propagation vs the oracle's FP64 propagation: |dP| <= 1e-12;
  * FP32 propagation vs FP64: |dP| <= 1e-5 (the target in the problem
    statement), typically ~1e-8;
  * full-size (n = 20, m = 4) runs: FP32 vs FP64 |dP| <= 1e-5, P in [0, 1].
"""
import os
import subprocess

import numpy as np
import pytest

from tests.conftest import load_golden

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n", [1, 2, 3, 5, 8, 10, 12, 13, 14, 16, 18, 20])
def test_diag_bit_exact(ctx, orc, n):
    for seed in (n, 1000 + n):
        raw = orc.sk_instances(n, 1, seed)[0]
        hp, E, info = ctx.build_diag(n, raw, energies=True)
        Eo, hpo, io = orc.energies_ref(n, raw)
        assert np.array_equal(E, Eo), n
        assert np.array_equal(hp.view(np.uint32), hpo.view(np.uint32)), n
        assert info.e_loc == io.e_loc
        assert info.e0 == io.e0 and info.emax == io.emax and info.mid == io.mid
        assert np.float32(info.e_abs) == np.float32(io.e_abs)


def test_diag_planted_tie_first_in_gray_order(ctx, orc):
    n = 9
    rng = np.random.default_rng(5)
    raw = np.zeros(n * (n + 1) // 2)
    raw[: n * (n - 1) // 2] = rng.integers(-8, 9, n * (n - 1) // 2) / 8.0
    _, E, info = ctx.build_diag(n, raw, energies=True)
    _, _, io = orc.energies_ref(n, raw)
    assert (E == E.min()).sum() >= 2
    assert info.e_loc == io.e_loc


def test_cheb_bit_exact(ctx, orc):
    s = np.array([1e-9, 2e-7, 1e-3, 0.37, 1.0, 3.3, 12.3, 37.0, 99.9, 150.0, 420.0, 901.5, 2500.0])
    coeffs, K = ctx.cheb_coeffs(s, max_k=4096)
    for i, sv in enumerate(s):
        ref = orc.cheb_coeffs(sv).astype(np.float32)
        assert K[i] == len(ref), sv
        assert np.array_equal(coeffs[i].view(np.uint32), ref.view(np.uint32)), sv


def _planar_to_complex(x):
    N = len(x) // 2
    return x[:N] + 1j * x[N:]


@pytest.mark.parametrize("n", [6, 9, 11, 12, 15, 17, 19, 21])
def test_clenshaw_single_propagation(ctx, orc, n):
    # n = 19: FP64 tiles span 2-CTA clusters; n = 21: FP32 2-CTA and FP64
    # 4-CTA clusters.
    N = 1 << n
    raw = orc.sk_instances(n, 1, 40 + n)[0]
    _, hp, info = orc.energies_ref(n, raw)
    g, _, t, _ = orc.schedule(n, 3, raw)
    rng = np.random.default_rng(n)
    psi = (rng.standard_normal(N) + 1j * rng.standard_normal(N)) / np.sqrt(2 * N)
    onenorm = float(np.float32(np.float32(info.e_abs) + np.float32(g[1]) * np.float32(n)))
    s = float(np.float32(np.float32(onenorm) * t[1, 3]))
    c = orc.cheb_coeffs(s).astype(np.float32)
    planar = np.concatenate([psi.real, psi.imag])
    ref64 = _planar_to_complex(orc.clenshaw(n, c, hp.astype(np.float64), float(g[1]), onenorm, planar, False, "f64"))
    out64 = ctx.clenshaw(n, c, hp, float(g[1]), onenorm, psi, "fp64")
    assert np.abs(out64 - ref64).max() < 1e-12
    out32 = ctx.clenshaw(n, c, hp, float(g[1]), onenorm, psi.astype(np.complex64), "fp32")
    err = np.linalg.norm(out32 - ref64) / np.linalg.norm(ref64)
    assert err < 2e-5, err


def test_config1_fp64_matches_oracle(ctx, orc):
    g = load_golden("oracle_config1.json")
    raw = orc.sk_instances(g["n"], g["count"], g["seed"])
    r = ctx.run_problems(g["n"], g["m"], raw, precision="fp64")
    assert r["e_loc"].tolist() == g["e_loc"]
    assert np.array_equal(r["total_t"], np.array(g["total_t"], np.float32))
    assert np.abs(r["p"] - np.array(g["p_f64"])).max() < 1e-12
    assert r["stats"]["terms"] == sum(g["terms"])


def test_config1_fp32_within_target(ctx, orc):
    g = load_golden("oracle_config1.json")
    raw = orc.sk_instances(g["n"], g["count"], g["seed"])
    r = ctx.run_problems(g["n"], g["m"], raw, precision="fp32")
    d64 = np.abs(r["p"] - np.array(g["p_f64"])).max()
    d32 = np.abs(r["p"] - np.array(g["p_f32"])).max()
    assert d64 <= 1e-5, d64
    assert d32 <= 1e-5, d32


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_small_cases_resident_and_grid(ctx, orc, precision):
    tol = 1e-12 if precision == "fp64" else 1e-5
    for c in load_golden("oracle_small.json")["cases"]:
        raw = orc.sk_instances(c["n"], c["count"], c["seed"])
        ref = np.array(c["p_f64"])
        for res in (0, -1):  # default (resident where it fits) / grid path only
            r = ctx.run_problems(c["n"], c["m"], raw, samples=c["samples"], precision=precision,
                                 resident_max_n=res)
            assert np.abs(r["p"] - ref).max() <= tol, (c["n"], c["m"], res)
            assert r["e_loc"].tolist() == c["e_loc"]


def test_mixed_plan_matches_single_runs(ctx, orc, mqw):
    ns = [6, 9, 12, 14, 6, 15]
    ms = [2, 3, 1, 2, 4, 3]
    raws = [orc.sk_instances(n, 1, 300 + i)[0] for i, (n, m) in enumerate(zip(ns, ms))]
    plan = mqw.Plan(ctx, ns, ms, np.concatenate(raws), samples=6, precision="fp64")
    plan.execute()
    res = plan.results()
    for i, (n, m) in enumerate(zip(ns, ms)):
        o = orc.run_problems(n, m, raws[i], 1, 6, "f64")
        assert abs(res["p"][i] - o["p"][0]) < 1e-12, (n, m)
    plan.close()


def test_plan_reexecute_is_deterministic(ctx, orc, mqw):
    raw = orc.sk_instances(15, 2, 4)
    plan = mqw.Plan(ctx, 15, 3, raw, samples=5)
    plan.execute()
    a = plan.results(per_sample=True)
    plan.execute()
    b = plan.results(per_sample=True)
    assert np.array_equal(a["p_sample"], b["p_sample"])
    plan.close()


def test_full_size_n20_m4_fp32_vs_fp64(ctx, orc):
    raw = orc.sk_instances(20, 1, 7)
    r32 = ctx.run_problems(20, 4, raw, samples=2, precision="fp32")
    r64 = ctx.run_problems(20, 4, raw, samples=2, precision="fp64")
    assert 0.0 <= r32["p"][0] <= 1.0
    assert abs(r32["p"][0] - r64["p"][0]) <= 1e-5
    _, _, io = orc.energies_ref(20, raw[0])
    assert r32["e_loc"][0] == io.e_loc


def test_cli_drop_in(ctx, orc, mqw, tmp_path):
    g = load_golden("oracle_config1.json")
    raw = orc.sk_instances(g["n"], 12, g["seed"])
    f = tmp_path / "SK_10n"
    raw.tofile(f)
    r = subprocess.run([mqw.CLI_PATH, "10", "2", str(f), "2", "7"], cwd=tmp_path,
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    lines = r.stdout.strip().splitlines()
    assert len(lines) == 7
    out = np.fromfile(tmp_path / "output_10_2", dtype=np.float32)
    ref = np.array(g["p_f64"][2:9])
    assert out.shape == (7,) and np.abs(out - ref).max() < 1e-5
    assert [float(x.split()[0]) for x in lines] == pytest.approx(g["total_t"][2:9], rel=1e-5)
    # appends, like the reference's ios::app
    r = subprocess.run([mqw.CLI_PATH, "10", "2", str(f), "0", "1"], cwd=tmp_path, capture_output=True)
    assert r.returncode == 0
    assert np.fromfile(tmp_path / "output_10_2", dtype=np.float32).shape == (8,)
    # a short file is an error, not a silent repeat
    r = subprocess.run([mqw.CLI_PATH, "10", "2", str(f), "10", "5"], cwd=tmp_path, capture_output=True)
    assert r.returncode == 1


def test_near_degenerate_n24_ground_state_index(ctx):
    """The 32 post-selected n = 24 instances (two lowest energies < 1e-2
    apart, two of them < 1e-4): the GPU diagonal gives the same ground-state
    index and the same gap as the oracle's reference-arithmetic screen."""
    from multistageqw_b200 import studies
    sel = load_golden("precision_n24_m4.json")
    for s in sel["instances"]:
        raw = studies.draw_raw(24, s["draw"])
        gap, e_loc, _ = studies.two_lowest_gap(ctx, 24, raw)
        assert e_loc == s["e_loc"], s
        assert gap == s["gap"], s


@pytest.mark.parametrize("n", [23, 25, 27])
def test_cluster_tiles_match_global_partner_path(ctx, orc, n):
    """Above n = 20 (FP32) the tiles span clusters of 4, 8 and 16 CTAs at
    n = 23, 25, 27. Capping the tile at 2^11 (tile_log = 11) instead runs the
    single-CTA path with the remaining axes read from global memory: both
    must agree with each other and with FP64 to the FP32 target."""
    raw = orc.sk_instances(n, 1, 500 + n)
    kw = dict(samples=1, graph=0, group=1)
    r_cl = ctx.run_problems(n, 2, raw, precision="fp32", **kw)
    r_gl = ctx.run_problems(n, 2, raw, precision="fp32", tile_log=11, **kw)
    r_64 = ctx.run_problems(n, 2, raw, precision="fp64", **kw)
    assert r_cl["stats"]["terms"] == r_gl["stats"]["terms"] == r_64["stats"]["terms"]
    assert abs(r_cl["p"][0] - r_gl["p"][0]) <= 1e-6
    assert abs(r_cl["p"][0] - r_64["p"][0]) <= 1e-5
    assert 0.0 < r_cl["p"][0] < 1.0


@pytest.mark.parametrize("n", [23, 25])
def test_single_cta_widest_tiles_match_cluster_tiles(ctx, orc, n):
    """cluster = -1 keeps the widest tile (2^12 in FP32) on one CTA and reads
    the axes neither tiling covers from global memory (3 at n = 23, 5 at
    n = 25) instead of spanning a cluster; with it the shared-basis chains
    run on the real chain kernel. Both shapes agree with each other and with
    FP64 to the FP32 target."""
    raw = orc.sk_instances(n, 1, 700 + n)
    kw = dict(samples=2, graph=0, group=1, tile_log=12)
    r_cl = ctx.run_problems(n, 2, raw, precision="fp32", cluster=1, **kw)
    r_gl = ctx.run_problems(n, 2, raw, precision="fp32", cluster=-1, **kw)
    r_64 = ctx.run_problems(n, 2, raw, precision="fp64", samples=2, graph=0)
    assert r_cl["stats"]["terms"] == r_gl["stats"]["terms"] == r_64["stats"]["terms"]
    assert abs(r_cl["p"][0] - r_gl["p"][0]) <= 1e-6
    assert abs(r_gl["p"][0] - r_64["p"][0]) <= 1e-5
    assert 0.0 < r_gl["p"][0] < 1.0


def test_lanes_give_identical_results(ctx, orc, mqw):
    """Walk groups run on 1, 2 or 3 concurrent lanes (streams, and branches
    of the captured graph) produce bit-identical per-sample results."""
    raw = orc.sk_instances(16, 3, 77)
    out = []
    for lanes in (1, 2, 3):
        plan = mqw.Plan(ctx, 16, 3, raw, samples=7, group=2, lanes=lanes)
        plan.execute()
        plan.execute()  # captures the graph
        plan.execute()  # graph replay
        out.append(plan.results(per_sample=True)["p_sample"])
        plan.close()
    assert np.array_equal(out[0], out[1]) and np.array_equal(out[0], out[2])


@pytest.mark.parametrize("n,m", [(14, 2), (17, 3), (20, 4)])
def test_stage1_basis_matches_per_walk_recurrence(ctx, orc, n, m):
    """The shared stage-1 basis (built once per instance, recombined per
    walk) against every walk running its own first-stage recurrence and
    against FP64: same ground-state probabilities to FP32 accuracy, with less
    pass work."""
    raw = orc.sk_instances(n, 2, 900 + n)
    kw = dict(samples=12, graph=0)
    on = ctx.run_problems(n, m, raw, precision="fp32", **kw)
    off = ctx.run_problems(n, m, raw, precision="fp32", stage1_basis=0, **kw)
    r64 = ctx.run_problems(n, m, raw, precision="fp64", **kw)
    assert np.abs(on["p"] - off["p"]).max() <= 1e-6
    assert np.abs(on["p"] - r64["p"]).max() <= 1e-5
    assert on["stats"]["term_amps"] == off["stats"]["term_amps"]
    assert on["stats"]["pass_amps"] < 0.95 * off["stats"]["pass_amps"]


@pytest.mark.parametrize("n", [19, 20])
@pytest.mark.parametrize("lane_smem", [-1, 1])
def test_256_thread_tiles_match_512(ctx, orc, n, lane_smem):
    """The widest FP32 tile with 256 threads (8 pairs per thread, P kept in
    registers) against 512 threads (4 pairs, P staged in shared memory), with
    the lane axes by shuffles (-1) or through shared memory (1), and all
    against FP64."""
    raw = orc.sk_instances(n, 1, 1300 + n)
    kw = dict(samples=6, graph=0, tile_log=12, group=2, lanes=1, resident_max_n=-1,
              lane_smem=lane_smem)
    r256 = ctx.run_problems(n, 3, raw, precision="fp32", threads=256, **kw)
    r512 = ctx.run_problems(n, 3, raw, precision="fp32", threads=512, **kw)
    r64 = ctx.run_problems(n, 3, raw, precision="fp64", samples=6, graph=0)
    assert abs(r256["p"][0] - r512["p"][0]) <= 1e-6
    assert abs(r256["p"][0] - r64["p"][0]) <= 1e-5


@pytest.mark.parametrize("n", [21, 24])
def test_wide_tile_2_13_matches(ctx, orc, n):
    """The 2^13-amplitude FP32 tile (8 pairs per thread, one CTA per SM)
    against the default tile and FP64."""
    raw = orc.sk_instances(n, 1, 1700 + n)
    kw = dict(samples=2, graph=0, group=1, lanes=1)
    r13 = ctx.run_problems(n, 2, raw, precision="fp32", tile_log=13, **kw)
    r13s = ctx.run_problems(n, 2, raw, precision="fp32", tile_log=13, lane_smem=1, **kw)
    assert abs(r13s["p"][0] - r13["p"][0]) <= 1e-6
    r12 = ctx.run_problems(n, 2, raw, precision="fp32", tile_log=12, **kw)
    r64 = ctx.run_problems(n, 2, raw, precision="fp64", samples=2, graph=0)
    assert abs(r13["p"][0] - r12["p"][0]) <= 1e-6
    assert abs(r13["p"][0] - r64["p"][0]) <= 1e-5


@pytest.mark.parametrize("n", [8, 15, 20])
def test_diag_moments(ctx, orc, n):
    """GPU moments of the shifted diagonal against numpy on the oracle's
    bit-identical diagonal (FP64 sums; relative 1e-12)."""
    raw = orc.sk_instances(n, 1, 2100 + n)[0]
    _, hp, _ = orc.energies_ref(n, raw)
    x = hp.astype(np.float64)
    ref = np.array([np.mean(x), np.mean(x ** 2), np.mean(x ** 3), np.mean(x ** 4)])
    m = ctx.diag_moments(n, raw)
    scale = np.array([np.sqrt(ref[1]), ref[1], ref[1] ** 1.5, ref[1] ** 2])
    assert np.all(np.abs(m - ref) <= 1e-12 * scale), (m, ref)
    assert np.array_equal(m, ctx.diag_moments(n, raw))  # deterministic


@pytest.mark.parametrize("n,tile", [(16, 0), (20, 12), (24, 11), (24, 13)])
def test_bulk_copy_staging_matches_cp_async(ctx, orc, n, tile):
    """Tiles staged by bulk copies on an mbarrier (TMA) against per-thread
    cp.async staging: the same arithmetic, so equal results up to nothing
    (bit-identical per-sample values), and within FP32 of FP64."""
    raw = orc.sk_instances(n, 1, 2500 + n)
    kw = dict(samples=3, graph=0, group=1, lanes=1, tile_log=tile, threads=512, lane_smem=-1,
              stage1_basis=0)
    r_t = ctx.run_problems(n, 2, raw, precision="fp32", tma=1, **kw)
    r_c = ctx.run_problems(n, 2, raw, precision="fp32", tma=-1, **kw)
    assert r_t["p"][0] == r_c["p"][0]
    r64 = ctx.run_problems(n, 2, raw, precision="fp64", samples=3, graph=0)
    assert abs(r_t["p"][0] - r64["p"][0]) <= 1e-5


def test_bounded_wait_reports_timeout_and_context_survives(ctx, orc, mqw):
    """A pass whose bulk copies can never complete (its mbarrier expects
    bytes nobody sends) gives up after its 5 ms bound, reports
    MQW_ERR_TIMEOUT through the device error word, and the context keeps
    working."""
    st = mqw.lib().mqw_selftest_wait_timeout(ctx.h)
    assert st == 5, st  # MQW_ERR_TIMEOUT
    raw = orc.sk_instances(14, 1, 3)
    r = ctx.run_problems(14, 2, raw, samples=2, tma=1)
    o = orc.run_problems(14, 2, raw, 1, 2, "f64")
    assert abs(r["p"][0] - o["p"][0]) <= 1e-5


@pytest.mark.parametrize("n", [14, 20, 22])
def test_compensated_fp32_is_closer_to_fp64(ctx, orc, n):
    """FP32 with compensated partner sums against plain FP32: both within the
    target of FP64, the compensated state closer to it."""
    raw = orc.sk_instances(n, 1, 2700 + n)[0]
    hp, _, info = ctx.build_diag(n, raw)
    g, _, t, _ = mqw_schedule(n, raw)
    N = 1 << n
    onenorm = float(np.float32(np.float32(info.e_abs) + np.float32(g[1]) * np.float32(n)))
    s = float(np.float32(np.float32(onenorm) * t[1, 7]))
    c = orc.cheb_coeffs(s).astype(np.float32)
    rng = np.random.default_rng(n)
    psi = ((rng.standard_normal(N) + 1j * rng.standard_normal(N)) / np.sqrt(2 * N))
    ref = ctx.clenshaw(n, c, hp, float(g[1]), onenorm, psi, "fp64")
    e32 = np.linalg.norm(ctx.clenshaw(n, c, hp, float(g[1]), onenorm, psi, "fp32") - ref)
    e32c = np.linalg.norm(ctx.clenshaw(n, c, hp, float(g[1]), onenorm, psi, "fp32c") - ref)
    nr = np.linalg.norm(ref)
    assert e32 / nr < 2e-5 and e32c / nr < 2e-5
    assert e32c < e32
    r = ctx.run_problems(n, 3, raw, samples=4, precision="fp32c", graph=0)
    r64 = ctx.run_problems(n, 3, raw, samples=4, precision="fp64", graph=0)
    assert abs(r["p"][0] - r64["p"][0]) <= 1e-5


def mqw_schedule(n, raw):
    import multistageqw_b200 as M
    return M.schedule(n, 3, raw)


def test_stage_scale_with_mixed_m(ctx, orc, mqw):
    """Per-stage (gamma, t) multipliers laid out instance after instance for a
    batch of different m: each instance gets its own, as when run alone."""
    ns, ms = [12, 14, 12], [2, 4, 3]
    raws = [orc.sk_instances(n, 1, 3100 + i)[0] for i, n in enumerate(ns)]
    rng = np.random.default_rng(5)
    scales = [rng.uniform(0.7, 1.4, (m, 2)).astype(np.float32) for m in ms]
    plan = mqw.Plan(ctx, ns, ms, np.concatenate(raws), samples=5,
                    stage_scale=np.concatenate(scales).ravel(), graph=0)
    plan.execute()
    p = plan.results()["p"]
    plan.close()
    for i, (n, m) in enumerate(zip(ns, ms)):
        r = ctx.run_problems(n, m, raws[i][None, :], samples=5, stage_scale=scales[i].ravel())
        assert abs(p[i] - r["p"][0]) <= 1e-6, i


def test_grid_shape_query(ctx):
    g = ctx.grid_shape(18)
    assert 6 <= g["tile_log"] <= 13 and g["group"] >= 1 and g["lanes"] >= 1
    assert g["threads"] in (256, 512) and g["us_per_walk_pass"] > 0
    assert ctx.grid_shape(18) == g  # cached per context


@pytest.mark.parametrize("n,m", [(15, 2), (17, 3), (20, 4), (22, 3)])
def test_final_projection_matches_per_walk_last_stage(ctx, orc, n, m):
    """The last stage as a projection onto the basis built from e_{E_loc}
    (output norm taken as the input norm) against every walk running its own
    last-stage recurrence and against FP64: per-sample P within 2e-6
    relative (the Chebyshev tail bound) plus FP32 rounding."""
    raw = orc.sk_instances(n, 1, 3300 + n)
    kw = dict(samples=8, graph=0)
    on = ctx.run_problems(n, m, raw, precision="fp32", **kw)
    off = ctx.run_problems(n, m, raw, precision="fp32", final_projection=0, **kw)
    r64 = ctx.run_problems(n, m, raw, precision="fp64", **kw)
    p_on, p_off = on["p"][0], off["p"][0]
    assert abs(p_on - p_off) <= 2e-6 * p_off + 1e-8, (p_on, p_off)
    assert abs(p_on - r64["p"][0]) <= 1e-5
    assert on["stats"]["pass_amps"] < off["stats"]["pass_amps"]
    plan = mqw_plan_samples(ctx, n, m, raw)
    assert np.all(plan >= 0.0) and np.all(plan <= 1.0)


def mqw_plan_samples(ctx, n, m, raw):
    import multistageqw_b200 as M
    plan = M.Plan(ctx, n, m, raw, samples=8)
    plan.execute()
    plan.execute()  # captures the graph
    plan.execute()  # graph replay
    ps = plan.results(per_sample=True)["p_sample"]
    plan.close()
    return ps


def test_basis_build_ahead_gives_identical_results(ctx, orc, mqw):
    """Building the next instance's bases on a side stream (MQW_BASIS_AHEAD=1,
    read once per process, so run in a child process) changes only the
    schedule: per-sample P bit-identical to the in-order build."""
    import json
    import sys
    raw = orc.sk_instances(16, 3, 4100)
    plan = mqw.Plan(ctx, 16, 3, raw, samples=6, group=1, lanes=2)
    plan.execute()
    plan.execute()
    ref = plan.results(per_sample=True)["p_sample"]
    plan.close()
    code = (
        "import json, numpy as np, multistageqw_b200 as M\n"
        "raw = M.sk_instances(16, 3, 4100)\n"
        "c = M.Context(0)\n"
        "pl = M.Plan(c, 16, 3, raw, samples=6, group=1, lanes=2)\n"
        "pl.execute(); pl.execute()\n"
        "print(json.dumps(pl.results(per_sample=True)['p_sample'].tolist()))\n")
    env = dict(os.environ, MQW_BASIS_AHEAD="1")
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, env=env,
                       cwd=os.path.dirname(os.path.dirname(os.path.abspath(__file__))), timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    got = np.array(json.loads(r.stdout.strip().splitlines()[-1]))
    assert np.array_equal(got, ref)


@pytest.mark.parametrize("n,m,samples", [(16, 3, 11), (20, 4, 8)])
def test_basis_groups_give_identical_results(ctx, orc, mqw, monkeypatch, n, m, samples):
    """The stage-1 recombination and the last-stage projection of a basis
    group of walks read each basis vector once for all of them; per walk the
    arithmetic is the one of a group of one (the FP32 sums in the same order;
    FP64 norms to within their rounding), so per-sample P matches basis groups
    of one walk (MQW_BASIS_GROUP=1, read at every plan) to 1e-12."""
    raw = orc.sk_instances(n, 1, 4200 + n)

    def run():
        plan = mqw.Plan(ctx, n, m, raw, samples=samples, group=1, lanes=2, graph=0)
        plan.execute()
        ps = plan.results(per_sample=True)["p_sample"]
        plan.close()
        return ps

    grouped = run()
    monkeypatch.setenv("MQW_BASIS_GROUP", "1")
    single = run()
    np.testing.assert_allclose(grouped, single, rtol=1e-12, atol=0.0)
    assert np.all(grouped > 0.0) and np.all(grouped <= 1.0)


@pytest.mark.parametrize("n,m,samples", [(16, 3, 24), (20, 4, 12), (18, 5, 16), (21, 3, 6),
                                          (14, 3, 100)])
def test_stage2_basis_matches_per_walk(ctx, orc, mqw, monkeypatch, n, m, samples):
    """Stage 2 from the product basis Y_jk = U_k(H~_2) w_j and one GEMM over
    the instance's walks (MQW_STAGE2_BASIS=1, read at every plan) against
    every walk running its own stage-1 recombination and stage-2 recurrence
    (=0): per-sample P within FP32 rounding, the mean within 1e-5 of FP64, and
    a captured graph replays it unchanged. n = 21 runs the chains with an
    axis read from global memory (double-buffered b, four walk slots); 100
    walks (the most an instance has) take the 128-column GEMM tile."""
    raw = orc.sk_instances(n, 1, 4400 + n)

    shape = {"tile_log": 12} if n > 20 else {}  # 2^12 tiles leave an axis to global memory

    def run(mode, graph):
        monkeypatch.setenv("MQW_STAGE2_BASIS", mode)
        plan = mqw.Plan(ctx, n, m, raw, samples=samples, graph=graph, **shape)
        plan.execute()
        first = plan.results(per_sample=True)["p_sample"]
        plan.execute()  # captures the graph (graph = 1)
        plan.execute()  # replays it
        again = plan.results(per_sample=True)["p_sample"]
        plan.close()
        return first, again

    on, on_replay = run("1", 1)
    off, _ = run("0", 0)
    assert np.array_equal(on, on_replay)
    np.testing.assert_allclose(on, off, rtol=5e-6, atol=1e-9)
    assert np.all(on > 0.0) and np.all(on <= 1.0)
    r64 = ctx.run_problems(n, m, raw, samples=samples, precision="fp64", graph=0)
    assert abs(float(np.mean(on)) - r64["p"][0]) <= 1e-5


def test_stage2_basis_in_a_mixed_m_plan(ctx, orc, mqw, monkeypatch):
    """One plan of instances of the same n with m = 3, 2, 4, 5 (the product
    basis used instance by instance where m >= 3, its buffers reused) and the
    learned-schedule hook (per-stage gamma/t multipliers) against the same
    plan with every walk running its own stage 2: per-sample P within FP32
    rounding."""
    ms = [3, 2, 4, 5]
    raws = np.concatenate([orc.sk_instances(16, 1, 4600 + i) for i in range(len(ms))])
    rng = np.random.default_rng(11)
    scale = rng.uniform(0.8, 1.25, (sum(ms), 2)).astype(np.float32).ravel()

    def run(mode):
        monkeypatch.setenv("MQW_STAGE2_BASIS", mode)
        plan = mqw.Plan(ctx, [16] * len(ms), ms, raws, samples=20, stage_scale=scale)
        plan.execute()
        plan.execute()
        ps = plan.results(per_sample=True)["p_sample"]
        st = plan.stats()
        plan.close()
        return ps, st

    on, st_on = run("1")
    off, st_off = run("0")
    np.testing.assert_allclose(on, off, rtol=5e-6, atol=1e-9)
    assert st_on["pass_amps"] != st_off["pass_amps"]


def test_stage2_basis_on_near_degenerate_instances(ctx, mqw, monkeypatch):
    """The stage-2 product basis where precision matters most: n = 20
    instances whose two lowest energies lie within 2e-2 (screened on the GPU
    from the precision study's seeded draws), per-sample P against FP64
    within the 1e-5 target and the mean far inside it."""
    from multistageqw_b200 import studies
    kept, seen, _ = studies.screen(ctx, 20, 2, 2e-2, 1500)
    assert len(kept) == 2, seen
    monkeypatch.setenv("MQW_STAGE2_BASIS", "1")
    for k in kept:
        raw = k["raw"][None, :]
        plan = mqw.Plan(ctx, 20, 4, raw, samples=24, graph=0)
        plan.execute()
        on = plan.results(per_sample=True)["p_sample"][0]
        plan.close()
        p64 = mqw.Plan(ctx, 20, 4, raw, samples=24, graph=0, precision="fp64")
        p64.execute()
        ref = p64.results(per_sample=True)["p_sample"][0]
        p64.close()
        assert np.max(np.abs(on - ref)) <= 1e-5, (k["gap"], np.max(np.abs(on - ref)))
        assert abs(on.mean() - ref.mean()) <= 1e-6


def test_stage2_basis_built_ahead_gives_identical_results(ctx, orc, mqw, monkeypatch):
    """The stage-2 product basis built on the build-ahead's side stream (its
    own chain slots, double-buffered Y and outputs; MQW_BASIS_AHEAD=1 is read
    once per process, so a child process) against the in-order build, over
    three instances: per-sample P equal to FP64 rounding."""
    import json
    import sys
    raws = np.concatenate([orc.sk_instances(16, 1, 4500 + i) for i in range(3)])
    monkeypatch.setenv("MQW_STAGE2_BASIS", "1")
    plan = mqw.Plan(ctx, 16, 3, raws, samples=12, group=1, lanes=2)
    plan.execute()
    plan.execute()
    ref = plan.results(per_sample=True)["p_sample"]
    plan.close()
    code = (
        "import json, numpy as np, multistageqw_b200 as M\n"
        "raws = np.concatenate([M.sk_instances(16, 1, 4500 + i) for i in range(3)])\n"
        "c = M.Context(0)\n"
        "pl = M.Plan(c, 16, 3, raws, samples=12, group=1, lanes=2)\n"
        "pl.execute(); pl.execute()\n"
        "print(json.dumps(pl.results(per_sample=True)['p_sample'].tolist()))\n")
    env = dict(os.environ, MQW_BASIS_AHEAD="1", MQW_STAGE2_BASIS="1")
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, env=env,
                       cwd=os.path.dirname(os.path.dirname(os.path.abspath(__file__))), timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    got = np.array(json.loads(r.stdout.strip().splitlines()[-1]))
    np.testing.assert_allclose(got, ref, rtol=1e-12, atol=0.0)


def test_tier_peaks(ctx):
    """The bandwidth probes: shared memory above L2 above HBM, HBM within
    reach of the B200's nominal 7.7 TB/s."""
    t = ctx.measure_peaks()
    assert 2000 < t["hbm_copy_gbs"] < 9000, t
    assert t["l2_read_gbs"] > t["hbm_copy_gbs"], t
    assert t["smem_gbs"] > t["l2_read_gbs"], t


def test_mixed_batch_per_instance_fp32_vs_fp64(ctx, mqw):
    """The mixed batch's first 16 instances (n in {12..20}, m in {2..5},
    drawn like the 4096-instance batch) as one FP32 plan at the full 100
    samples, every instance within 1e-5 of the same plan in FP64, with the
    same ground-state index; the draw covers n = 18 and 20 and m = 5."""
    from multistageqw_b200 import studies
    ns, ms, raw = studies.mixed_batch(16, 0)
    assert {18, 20} <= set(ns) and max(ms) == 5
    out = {}
    for prec in ("fp32", "fp64"):
        plan = mqw.Plan(ctx, ns, ms, raw, samples=100, precision=prec, graph=0)
        plan.execute()
        out[prec] = plan.results()
        plan.close()
    dP = np.abs(out["fp32"]["p"] - out["fp64"]["p"])
    assert dP.max() <= 1e-5, dP
    assert out["fp32"]["e_loc"].tolist() == out["fp64"]["e_loc"].tolist()


def test_n28_m3_fp32_vs_fp64(ctx, orc):
    """The largest size, n = 28 (2^28 amplitudes, tiles over clusters or
    with global-memory axes), m = 3, one sample of the seed-7 instance: FP32
    within 1e-5 of FP64 and the reference-arithmetic ground-state index."""
    raw = orc.sk_instances(28, 1, 7)
    r32 = ctx.run_problems(28, 3, raw, samples=1, precision="fp32")
    r64 = ctx.run_problems(28, 3, raw, samples=1, precision="fp64")
    assert 0.0 <= r32["p"][0] <= 1.0
    assert abs(r32["p"][0] - r64["p"][0]) <= 1e-5
    assert r32["e_loc"][0] == r64["e_loc"][0]


def test_run_driver_output_is_in_problem_order(mqw, orc, tmp_path):
    """The run.sh-compatible driver over 4 concurrent ranges writes
    output_<n>_<m> byte-identical to one MultiQW run over the whole range
    (problem order, not completion order), for every (n, m) of its lists,
    and appends like the reference."""
    import os
    raw = orc.sk_instances(7, 23, 5)
    (tmp_path / "SK_7n").write_bytes(raw.tobytes())
    single = tmp_path / "single"
    single.mkdir()
    for m in (1, 3):
        r = subprocess.run([mqw.CLI_PATH, "7", str(m), str(tmp_path / "SK_7n"), "0", "23"],
                           cwd=single, capture_output=True, text=True)
        assert r.returncode == 0, r.stderr
    script = os.path.join(os.path.dirname(mqw.LIB_PATH), "..", "run.sh")
    env = dict(os.environ, MQW_N_VALUES="7", MQW_M_VALUES="1 3", MQW_PROBLEMS="23")
    for _ in range(2):  # the second run appends
        r = subprocess.run(["bash", script, "4", "SK"], cwd=tmp_path, env=env,
                           capture_output=True, text=True)
        assert r.returncode == 0, r.stderr
        assert len(r.stdout.strip().splitlines()) == 46
    for m in (1, 3):
        a = (single / f"output_7_{m}").read_bytes()
        assert len(a) == 23 * 4
        assert (tmp_path / f"output_7_{m}").read_bytes() == a + a


@pytest.mark.parametrize("n,m,samples", [(16, 3, 24), (20, 4, 100), (14, 5, 7)])
def test_stage2_tensor_core_gemm_matches_simt(ctx, orc, mqw, monkeypatch, n, m, samples):
    """The stage-2 product-basis GEMM on the tensor cores (tcgen05 kind::tf32
    with the three-product TF32 split, the default) against the FP32 SIMT
    GEMM (MQW_S2_GEMM=simt) on the same product basis: per-sample P within
    FP32-level rounding (5e-6 relative), the mean within 1e-5 of FP64; 7
    walks take a 16-column MMA, 100 walks a 112-column one."""
    raw = orc.sk_instances(n, 1, 5100 + n)
    monkeypatch.setenv("MQW_STAGE2_BASIS", "1")

    def run(gemm):
        if gemm:
            monkeypatch.setenv("MQW_S2_GEMM", gemm)
        else:
            monkeypatch.delenv("MQW_S2_GEMM", raising=False)
        plan = mqw.Plan(ctx, n, m, raw, samples=samples, graph=0)
        plan.execute()
        out = plan.results(per_sample=True)["p_sample"]
        plan.close()
        return out

    tc = run(None)
    simt = run("simt")
    np.testing.assert_allclose(tc, simt, rtol=5e-6, atol=1e-9)
    r64 = ctx.run_problems(n, m, raw, samples=samples, precision="fp64", graph=0)
    assert abs(float(np.mean(tc)) - r64["p"][0]) <= 1e-5


@pytest.mark.parametrize("n,tile,threads", [(19, 12, 256), (20, 12, 256), (22, 13, 512),
                                            (24, 13, 512)])
def test_second_exchange_tile_matches_one(ctx, orc, n, tile, threads):
    """A second exchange tile (tma=2, shapes with 8 pairs per thread: the
    256-thread 2^12 tile and the 2^13 tile) against the single tile: the same
    arithmetic, so bit-identical per-sample values, including n = 24 (2^13
    tiles, two axes read from global memory), and within FP32 of FP64."""
    raw = orc.sk_instances(n, 1, 2700 + n)
    kw = dict(samples=3, graph=0, group=1, lanes=1, tile_log=tile, threads=threads, lane_smem=-1,
              stage1_basis=0)
    r_d = ctx.run_problems(n, 3, raw, precision="fp32", tma=2, **kw)
    r_c = ctx.run_problems(n, 3, raw, precision="fp32", tma=-1, **kw)
    assert r_d["p"][0] == r_c["p"][0]
    r64 = ctx.run_problems(n, 3, raw, precision="fp64", samples=3, graph=0)
    assert abs(r_d["p"][0] - r64["p"][0]) <= 1e-5


def test_each_device_gets_its_own_shared_memory_opt_in(mqw, orc):
    """Kernels above 48 KB of shared memory are opted in per device: after
    FP32 and FP64 runs on device 0 the same runs on device 1 (a second
    context in the same process) must launch too and agree. Needs two GPUs;
    skipped otherwise."""
    import torch
    if torch.cuda.device_count() < 2:
        pytest.skip("needs two GPUs")
    n = 16
    raw = orc.sk_instances(n, 1, 77)
    out = []
    for dev in (0, 1):
        c = mqw.Context(dev)
        out.append([c.run_problems(n, 3, raw, samples=4, precision=p)["p"][0]
                    for p in ("fp32", "fp64")])
        c.close()
    assert out[0] == out[1]


@pytest.mark.parametrize("n,m,samples,tile", [(16, 3, 24, 0), (20, 4, 12, 0), (21, 3, 6, 11),
                                              (14, 4, 9, 0)])
def test_real_chains_match_complex_chains(ctx, orc, mqw, monkeypatch, n, m, samples, tile):
    """The shared-basis chains on the real chain kernel (the default) against
    the same chains on the complex pass kernel (MQW_REAL_CHAINS=0): the real
    kernel reproduces the real parts bit for bit, so every per-sample P is
    identical — with the stage-2 product basis forced on (its chains start
    from the stage-1 basis vectors), and at n = 21 with 2^11 tiles, where
    three axes of every pass are read from global memory."""
    raw = orc.sk_instances(n, 1, 5300 + n)
    monkeypatch.setenv("MQW_STAGE2_BASIS", "1")
    # one launch per pass on both kernels (the same tiles; chain launches
    # are compared with single-pass launches in their own test)
    monkeypatch.setenv("MQW_CHAIN", "0")
    shape = {"tile_log": tile} if tile else {}

    def run(real):
        monkeypatch.setenv("MQW_REAL_CHAINS", "1" if real else "0")
        plan = mqw.Plan(ctx, n, m, raw, samples=samples, graph=0, **shape)
        plan.execute()
        out = plan.results(per_sample=True)["p_sample"]
        plan.close()
        return out

    on, off = run(True), run(False)
    assert np.array_equal(on, off)
    r64 = ctx.run_problems(n, m, raw, samples=samples, precision="fp64", graph=0)
    assert abs(float(np.mean(on)) - r64["p"][0]) <= 1e-5


@pytest.mark.parametrize("n,m,precision,s2", [(13, 3, "fp32", "-1"), (13, 2, "fp64", "-1"),
                                              (14, 3, "fp32", "-1"), (15, 4, "fp32", "-1"),
                                              (16, 3, "fp32", "-1"), (15, 2, "fp64", "-1"),
                                              (13, 4, "fp32", "1"), (16, 3, "fp32", "1")])
def test_chain_launch_matches_single_pass_launches(ctx, orc, mqw, monkeypatch, n, m, precision,
                                                   s2):
    """Small n: every term of a walk-stage in one launch (a thread-block
    cluster of up to 16 CTAs per walk, cluster barriers between the passes)
    against one launch per term (MQW_CHAIN=0), with a fraction of the
    launches. At n = 13 both use 16 tiles of 2^9 per walk, so the passes are
    the same arithmetic in the same order and every per-sample P is
    identical; above it the chain launch uses wider tiles (at most 16 per
    walk) than the single-pass launches, which changes the order of the
    partner sums, so per-sample P agree to FP32 (FP64) rounding. The grid
    path is forced (resident_max_n = -1) so that n = 13 takes it too. With
    the stage-2 product basis forced on (s2 = "1"), its chains run batched,
    one cluster per chain in one launch."""
    raw = orc.sk_instances(n, 2, 6100 + n)
    monkeypatch.setenv("MQW_STAGE2_BASIS", s2)

    def run(chain):
        monkeypatch.setenv("MQW_CHAIN", "1" if chain else "0")
        plan = mqw.Plan(ctx, n, m, raw, samples=8, graph=0, precision=precision,
                        resident_max_n=-1)
        plan.execute()
        out = plan.results(per_sample=True)["p_sample"]
        launches = plan.stats()["launches"]
        plan.close()
        return out, launches

    (on, l_on), (off, l_off) = run(True), run(False)
    if n == 13:
        assert np.array_equal(on, off)
    else:
        assert np.abs(on - off).max() <= (1e-7 if precision == "fp32" else 1e-13)
    assert l_on * 4 < l_off, (l_on, l_off)
    r64 = ctx.run_problems(n, m, raw, samples=8, precision="fp64", graph=0)
    assert np.abs(np.mean(on, axis=1) - r64["p"]).max() <= 1e-5


@pytest.mark.parametrize("n,m,samples,tile", [(18, 3, 40, 0), (21, 3, 12, 0), (20, 4, 24, 11)])
def test_batched_chain_passes_match_one_chain_per_launch(ctx, orc, mqw, monkeypatch, n, m,
                                                         samples, tile):
    """The stage-2 product basis's chains with up to 8 chains per launch
    (MQW_CHAIN_BATCH=8, each chain its own partial P) against one chain per
    launch: the same real passes on the same tiles, so every per-sample P is
    identical — at n = 21 and with 2^11 tiles at n = 20 with axes read from
    global memory."""
    raw = orc.sk_instances(n, 1, 7700 + n)
    monkeypatch.setenv("MQW_STAGE2_BASIS", "1")
    shape = {"tile_log": tile} if tile else {}

    def run(batch):
        monkeypatch.setenv("MQW_CHAIN_BATCH", str(batch))
        plan = mqw.Plan(ctx, n, m, raw, samples=samples, graph=0, **shape)
        plan.execute()
        out = plan.results(per_sample=True)["p_sample"]
        launches = plan.stats()["launches"]
        plan.close()
        return out, launches

    (on, l_on), (off, l_off) = run(8), run(1)
    assert np.array_equal(on, off)
    assert l_on < l_off


@pytest.mark.parametrize("n,samples", [(14, 40), (16, 24), (18, 16), (20, 100)])
def test_last_two_stage_basis_matches_recurrence(ctx, orc, mqw, monkeypatch, n, samples):
    """m = 4 with the product basis of the last two stages (MQW_LAST2_BASIS=1:
    chains U_k(H~_3) w'_j from the last-stage basis w'_j = U_j(H~_4) e_{E_loc},
    one GEMM for every walk's recombined vector, one bilinear sum with the
    walk's stage-2 state) against the stage-3 recurrence per walk and the
    last-stage projection (MQW_LAST2_BASIS=0). Both take a stage's output
    norm as its input norm only where the Chebyshev tail (1e-6) allows it,
    so per-sample P agree to a few 1e-6 relative; both within 1e-5 of FP64."""
    raw = orc.sk_instances(n, 1, 8800 + n)
    monkeypatch.setenv("MQW_STAGE2_BASIS", "1")

    def run(mode):
        monkeypatch.setenv("MQW_LAST2_BASIS", mode)
        plan = mqw.Plan(ctx, n, 4, raw, samples=samples, graph=0)
        plan.execute()
        out = plan.results(per_sample=True)["p_sample"]
        pass_amps = plan.stats()["pass_amps"]
        plan.close()
        return out, pass_amps

    (on, a_on), (off, a_off) = run("1"), run("0")
    assert np.all(np.abs(on - off) <= 1e-5 * np.abs(off) + 1e-10), np.abs(on / off - 1).max()
    assert a_on == 0 < a_off  # no walk ran a recurrence
    r64 = ctx.run_problems(n, 4, raw, samples=samples, precision="fp64", graph=0)
    assert abs(float(np.mean(on)) - r64["p"][0]) <= 1e-5


@pytest.mark.parametrize("n,m,samples", [(20, 4, 24), (19, 3, 20)])
def test_chain_lanes_do_not_change_results(ctx, orc, mqw, monkeypatch, n, m, samples):
    """The one-chain-per-launch product-basis chains run on four lanes from
    n = 19 (their slots packed in the state buffer); the lanes only reorder
    independent chains, so one lane (MQW_CHAIN_LANES=1) and seven give every
    per-sample P bit for bit as the default."""
    raw = orc.sk_instances(n, 1, 9100 + n)
    monkeypatch.setenv("MQW_STAGE2_BASIS", "1")

    def run(lanes):
        if lanes:
            monkeypatch.setenv("MQW_CHAIN_LANES", str(lanes))
        else:
            monkeypatch.delenv("MQW_CHAIN_LANES", raising=False)
        plan = mqw.Plan(ctx, n, m, raw, samples=samples, graph=0)
        plan.execute()
        out = plan.results(per_sample=True)["p_sample"]
        plan.close()
        return out

    ref = run(None)
    for lanes in (1, 7):
        assert np.array_equal(run(lanes), ref), lanes


_THREADS_SCRIPT = r"""
import sys
import numpy as np
sys.path.insert(0, sys.argv[1])
import multistageqw_b200 as M
out = []
for n, m in ((20, 4), (18, 3)):
    raw = M.sk_instances(n, 1, 9300 + n)
    ctx = M.Context(0)
    plan = M.Plan(ctx, n, m, raw, samples=12, graph=0)
    plan.execute()
    out.append(plan.results(per_sample=True)["p_sample"])
    plan.close()
    ctx.close()
np.save(sys.argv[2], np.concatenate([o.ravel() for o in out]))
"""


def test_real_pass_thread_counts_give_identical_results(mqw, tmp_path):
    """The real chain passes with 128, 256 (the defaults by tile) and 512
    or 1024 threads per CTA (MQW_REAL_THREADS, read once per process, so
    each runs in its own process) sum every partner in the same order:
    per-sample P bit for bit alike at n = 20 (2^12 tiles) and n = 18
    (2^11 tiles, eight chains per launch)."""
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(mqw.__file__)))
    script = tmp_path / "threads.py"
    script.write_text(_THREADS_SCRIPT)
    res = {}
    for t in ("", "128", "256", "512", "1024"):
        env = dict(os.environ)
        env.pop("MQW_REAL_THREADS", None)
        if t:
            env["MQW_REAL_THREADS"] = t
        out = tmp_path / f"p_{t or 'default'}.npy"
        r = subprocess.run([sys.executable, str(script), root, str(out)], env=env,
                           capture_output=True, text=True, timeout=600)
        assert r.returncode == 0, r.stderr[-2000:]
        res[t] = np.load(out)
    for t, v in res.items():
        assert np.array_equal(v, res[""]), t


def test_chain_pass_timing_mirrors_the_plans_launches(ctx):
    """mqw_chain_pass_timing launches what a plan launches: eight chains per
    launch at n = 18, one per launch on four lanes at n = 20."""
    t18 = ctx.chain_pass_timing(18, reps=8)
    t20 = ctx.chain_pass_timing(20, reps=8)
    assert t18["walks_per_launch"] == 8 and t18["us_per_launch"] > 0
    assert t20["walks_per_launch"] == 1 and t20["lanes"] == 4 and t20["us_per_launch"] > 0
