"""The learned stage schedule: MLP kernels against the float64 oracle, the
optimizer, features, the equal-cost rule, and the trained network's gain
over the plain heuristic."""
import os

import numpy as np
import pytest

from oracle import mlp_oracle as MO


def _params(rng, dims):
    return [(rng.standard_normal((dims[i + 1], dims[i])).astype(np.float32) / np.sqrt(dims[i]),
             rng.standard_normal(dims[i + 1]).astype(np.float32) * 0.1) for i in range(len(dims) - 1)]


def test_oracle_gradients_match_finite_differences():
    # Pins the oracle itself: analytic float64 gradients vs central differences
    # of the loss (weights fixed at their bfloat16 values, so the rounding is
    # not differentiated).
    rng = np.random.default_rng(0)
    dims = [5, 7, 6, 2]
    params = [(MO.bf16_round(W), b) for W, b in _params(rng, dims)]
    X = rng.standard_normal((9, 5))
    T = rng.standard_normal((9, 2))
    loss, grads = MO.mlp_loss_grad(params, X, T)
    eps = 1e-6
    for li, (W, b) in enumerate(params):
        Wd = W.astype(np.float64)
        for (i, j) in [(0, 0), (1, 2), (W.shape[0] - 1, W.shape[1] - 1)]:
            def f(delta):
                Wp = Wd.copy()
                Wp[i, j] += delta
                ps = list(params)
                ps[li] = (Wp, b)
                # bypass rounding for the perturbed weight: evaluate in float64
                acts = np.asarray(X, np.float64)
                for k, (Wk, bk) in enumerate(ps):
                    Z = acts @ np.asarray(Wk, np.float64).T + bk
                    acts = np.maximum(Z, 0) if k < len(ps) - 1 else Z
                return 0.5 * np.sum((acts - T) ** 2) / X.shape[0]
            num = (f(eps) - f(-eps)) / (2 * eps)
            assert abs(num - grads[li][0][i, j]) < 1e-6 * max(1.0, abs(num))


def test_features(mqw):
    from multistageqw_b200 import learned as LR
    raw = mqw.sk_instances(12, 1, 3)[0]
    f = LR.instance_features(12, 4, raw)
    assert f.shape == (4, LR.N_FEATURES)
    assert np.allclose(f[:, 1], [0, 1 / 3, 2 / 3, 1])
    assert np.all(f[:, 0] == 12 / 20) and np.all(f[:, 2] == 4 / 5)
    assert np.all(np.diff(f[0, 8:12]) <= 0)  # eigenvalues in decreasing order


def test_equal_cost_scale(mqw):
    from multistageqw_b200 import learned as LR
    n, m = 12, 4
    raw = mqw.sk_instances(n, 1, 5)[0]
    g, st, _, _ = mqw.schedule(n, m, raw)
    e_abs = 17.5
    rng = np.random.default_rng(1)
    for _ in range(5):
        dlg, dlt = rng.uniform(-0.5, 0.5, m), rng.uniform(-0.5, 0.5, m)
        sc = LR.equal_cost_scale(n, g, st, e_abs, dlg, dlt)
        c0 = np.sum((e_abs + g.astype(np.float64) * n) * st)
        c1 = np.sum((e_abs + sc[:, 0] * g * n) * sc[:, 1] * st)
        assert abs(c1 / c0 - 1) < 1e-5
    one = LR.equal_cost_scale(n, g, st, e_abs, np.zeros(m), np.zeros(m))
    assert np.allclose(one, 1.0)


@pytest.mark.gpu
def test_linear_kernels_match_oracle(mqw):
    import torch
    from multistageqw_b200 import learned as LR
    net = LR.StageMLP(0, seed=3)
    rng = np.random.default_rng(4)
    X = rng.standard_normal((37, LR.N_FEATURES)).astype(np.float32)
    T = rng.standard_normal((37, 2)).astype(np.float32)
    Y, acts = net.forward(torch.from_numpy(X).cuda())
    params = [(w.cpu().numpy(), b.cpu().numpy()) for w, b in zip(net.w, net.b)]
    Yo, acts_o = MO.mlp_forward(params, X)
    assert np.abs(Y.cpu().numpy() - Yo).max() < 1e-4 * max(1.0, np.abs(Yo).max())
    B = X.shape[0]
    dY = (Y - torch.from_numpy(T).cuda()) / B
    dWs, dbs = net.backward(acts, dY)
    # oracle gradients through the same (GPU-produced) activations' masks
    _, grads = MO.mlp_loss_grad(params, X, T)
    for li in range(len(params)):
        gw, gb = grads[li]
        assert np.abs(dWs[li].cpu().numpy() - gw).max() < 2e-4 * max(1e-3, np.abs(gw).max()), li
        assert np.abs(dbs[li].cpu().numpy() - gb).max() < 2e-4 * max(1e-3, np.abs(gb).max()), li


@pytest.mark.gpu
def test_adam_step_matches_numpy(mqw):
    import ctypes
    import torch
    rng = np.random.default_rng(2)
    w = rng.standard_normal(1000).astype(np.float32)
    g = rng.standard_normal(1000).astype(np.float32)
    dw, dg = torch.from_numpy(w.copy()).cuda(), torch.from_numpy(g).cuda()
    dm, dv = torch.zeros(1000, device="cuda"), torch.zeros(1000, device="cuda")
    wb = torch.empty(1000, dtype=torch.bfloat16, device="cuda")
    st = mqw.lib().mqw_mlp_adam(1000, ctypes.c_void_p(dw.data_ptr()), ctypes.c_void_p(wb.data_ptr()),
                                ctypes.c_void_p(dg.data_ptr()), ctypes.c_void_p(dm.data_ptr()),
                                ctypes.c_void_p(dv.data_ptr()), 1e-2, 0.9, 0.999, 1e-8, 0.0, 1, None)
    assert st == 0
    torch.cuda.synchronize()
    m = 0.1 * g
    v = 0.001 * g * g
    ref = w - 1e-2 * (m / 0.1) / (np.sqrt(v / 0.001) + 1e-8)
    assert np.abs(dw.cpu().numpy() - ref).max() < 1e-6
    assert np.array_equal(wb.float().cpu().numpy(), MO.bf16_round(dw.cpu().numpy()))


@pytest.mark.gpu
def test_training_fits_a_smooth_target(mqw):
    from multistageqw_b200 import learned as LR
    rng = np.random.default_rng(7)
    X = rng.standard_normal((2048, LR.N_FEATURES)).astype(np.float32)
    T = np.stack([np.tanh(X[:, 0] - 0.5 * X[:, 3]), 0.3 * np.sin(X[:, 1])], axis=1).astype(np.float32)
    net = LR.StageMLP(0, seed=1)
    losses = LR.train(net, X, T, steps=600, batch=256, lr=2e-3, log=None)
    assert losses[-1] < 0.1 * losses[0]


@pytest.mark.gpu
def test_learned_schedule_beats_heuristic_at_equal_cost(mqw):
    """The trained network (committed weights) against the plain heuristic on
    fresh instances from the training range, at equal simulated cost."""
    from multistageqw_b200 import learned as LR
    assert os.path.exists(LR.DEFAULT_MODEL), "trained model missing"
    ctx = mqw.Context(0)
    net = LR.StageMLP.load(LR.DEFAULT_MODEL)
    r = LR.evaluate(ctx, net, 14, 4, 48, 99001, samples=50)
    assert r["mean_p_learned"] > r["mean_p_heuristic"], r
    assert abs(r["terms_learned"] / r["terms_heuristic"] - 1) < 0.05, r
    # no model: the plain heuristic, exactly
    raws = mqw.sk_instances(12, 2, 5)
    assert np.all(LR.propose_stage_scale(ctx, None, 12, 3, raws) == 1.0)
    ctx.close()
