"""Learned per-stage (gamma, t) corrections on top of the paper heuristic.

The reference chooses each stage's hopping rate gamma_i and time scale t_i by
closed-form heuristics (MultiQW.cpp:365-422). Here a small MLP maps instance
and stage features to multiplicative corrections exp(dlog_gamma_i),
exp(dlog_t_i). It is trained on (gamma, t) scans generated by the simulator
itself, evaluated by the simulator's own ground-state probability, and
applied at equal simulated cost; the plain heuristic is the fallback whenever
no model is loaded or a proposal is not finite.

Network: 12 features -> 3 hidden layers of 256 (ReLU) -> 2 outputs, weights
stored in BF16, activations and accumulation in FP32, trained with Adam on
FP32 master weights. Forward, backward and the optimizer step are the
project's CUDA kernels (include/mqw.h, mqw_mlp_*); torch only holds device
memory.

Features of stage i of an instance (n spins, m stages):
    n/20, i/max(m-1, 1), m/5, mean J, std J, max |J|, mean |h|, std h,
    the four largest eigenvalues of the coupling matrix J divided by sqrt(n)
(J_ij over pairs i > j as stored in the instance file; eigenvalues in FP64
on the host).

Equal cost: a stage costs about s_i = onenorm_i * t_i Chebyshev terms per
sample (onenorm_i = E_abs + gamma_i n). Proposed time multipliers are rescaled
by one common factor so that sum_i onenorm_i' t_i' equals the heuristic's
sum_i onenorm_i t_i; the measured number of terms is reported for both.
"""
from __future__ import annotations

import ctypes
import json
import os
import time

import numpy as np

from . import Context, Plan, lib, schedule, sk_instances

N_FEATURES = 12
HIDDEN = 256
N_HIDDEN_LAYERS = 3
CLIP = 0.7  # |dlog| bound on proposals (multipliers within [0.5, 2])
DEFAULT_MODEL = os.path.join(os.path.dirname(os.path.abspath(__file__)), "models", "stage_mlp.npz")


# ---- features and equal-cost application -----------------------------------

def instance_features(n: int, m: int, raw: np.ndarray) -> np.ndarray:
    """[m, 12] float32 feature rows, one per stage."""
    raw = np.asarray(raw, np.float64)
    npair = n * (n - 1) // 2
    jp = raw[:npair]
    h = raw[npair:npair + n]
    J = np.zeros((n, n))
    k = 0
    for i in range(1, n):
        J[i, :i] = jp[k:k + i]
        k += i
    J = J + J.T
    ev = np.sort(np.linalg.eigvalsh(J))[::-1] / np.sqrt(n)
    top = np.zeros(4)
    top[:min(4, n)] = ev[:4]
    base = [n / 20.0, 0.0, m / 5.0,
            float(jp.mean()) if npair else 0.0, float(jp.std()) if npair else 0.0,
            float(np.abs(jp).max()) if npair else 0.0,
            float(np.abs(h).mean()), float(h.std())] + list(top)
    rows = np.tile(np.array(base, np.float32), (m, 1))
    rows[:, 1] = np.arange(m) / max(m - 1, 1)
    return rows


def equal_cost_scale(n: int, gammas, short_t, e_abs: float, dlg, dlt) -> np.ndarray:
    """[m, 2] multipliers (gamma, t) from log-corrections, with the time
    multipliers rescaled so the proposal costs what the heuristic costs."""
    gammas = np.asarray(gammas, np.float64)
    short_t = np.asarray(short_t, np.float64)
    fg = np.exp(np.clip(np.asarray(dlg, np.float64), -CLIP, CLIP))
    ft = np.exp(np.clip(np.asarray(dlt, np.float64), -CLIP, CLIP))
    on0 = e_abs + gammas * n
    on1 = e_abs + fg * gammas * n
    lam = float(np.sum(on0 * short_t) / np.sum(on1 * ft * short_t))
    return np.stack([fg, ft * lam], axis=1).astype(np.float32)


# ---- the network -------------------------------------------------------------

def _ck(status: int, what: str) -> None:
    if status != 0:
        raise RuntimeError(f"{what} failed with status {status}")


class StageMLP:
    """12 -> 256 -> 256 -> 256 -> 2 MLP on the GPU (BF16 weights, FP32 math)."""

    def __init__(self, device: int = 0, seed: int = 0):
        import torch
        self.torch = torch
        self.dev = torch.device("cuda", device)
        g = torch.Generator().manual_seed(seed)
        dims = [N_FEATURES] + [HIDDEN] * N_HIDDEN_LAYERS + [2]
        self.dims = dims
        self.w, self.b = [], []
        for i in range(len(dims) - 1):
            fan_in = dims[i]
            std = (2.0 / fan_in) ** 0.5 if i < len(dims) - 2 else 0.01
            self.w.append((torch.randn(dims[i + 1], dims[i], generator=g) * std).to(self.dev))
            self.b.append(torch.zeros(dims[i + 1], device=self.dev))
        self.wb = [torch.empty(w.shape, dtype=torch.bfloat16, device=self.dev) for w in self.w]
        self.m = [torch.zeros_like(t) for t in self.w + self.b]
        self.v = [torch.zeros_like(t) for t in self.w + self.b]
        self.step_count = 0
        self.feat_mean = np.zeros(N_FEATURES, np.float32)
        self.feat_std = np.ones(N_FEATURES, np.float32)
        self._refresh_bf16()

    def _stream(self):
        return ctypes.c_void_p(self.torch.cuda.current_stream(self.dev).cuda_stream)

    def _refresh_bf16(self):
        for w, wb in zip(self.w, self.wb):
            _ck(lib().mqw_mlp_to_bf16(w.numel(), ctypes.c_void_p(w.data_ptr()),
                                      ctypes.c_void_p(wb.data_ptr()), self._stream()), "to_bf16")

    def forward(self, X):
        """X: [B, 12] standardised device tensor -> (Y [B, 2], activations)."""
        acts = [X.contiguous()]
        L = len(self.w)
        for i in range(L):
            out = self.torch.empty(X.shape[0], self.dims[i + 1], device=self.dev)
            _ck(lib().mqw_mlp_linear_forward(
                X.shape[0], self.dims[i], self.dims[i + 1], ctypes.c_void_p(self.wb[i].data_ptr()),
                ctypes.c_void_p(self.b[i].data_ptr()), ctypes.c_void_p(acts[-1].data_ptr()),
                ctypes.c_void_p(out.data_ptr()), int(i < L - 1), self._stream()), "linear_forward")
            acts.append(out)
        return acts[-1], acts

    def backward(self, acts, dY):
        """Gradients (dW list, db list) of the loss whose output gradient is dY."""
        L = len(self.w)
        dWs, dbs = [None] * L, [None] * L
        d = dY.contiguous()
        for i in range(L - 1, -1, -1):
            dW = self.torch.empty_like(self.w[i])
            db = self.torch.empty_like(self.b[i])
            dX = self.torch.empty_like(acts[i]) if i > 0 else None
            _ck(lib().mqw_mlp_linear_backward(
                d.shape[0], self.dims[i], self.dims[i + 1], ctypes.c_void_p(self.wb[i].data_ptr()),
                ctypes.c_void_p(acts[i].data_ptr()), ctypes.c_void_p(acts[i + 1].data_ptr()),
                ctypes.c_void_p(d.data_ptr()), ctypes.c_void_p(dX.data_ptr()) if dX is not None else None,
                ctypes.c_void_p(dW.data_ptr()), ctypes.c_void_p(db.data_ptr()), int(i < L - 1),
                self._stream()), "linear_backward")
            dWs[i], dbs[i] = dW, db
            d = dX
        return dWs, dbs

    def adam(self, dWs, dbs, lr=1e-3, beta1=0.9, beta2=0.999, eps=1e-8, weight_decay=0.0):
        self.step_count += 1
        params = self.w + self.b
        grads = dWs + dbs
        for k, (p, g) in enumerate(zip(params, grads)):
            wb = self.wb[k] if k < len(self.w) else None
            _ck(lib().mqw_mlp_adam(p.numel(), ctypes.c_void_p(p.data_ptr()),
                                   ctypes.c_void_p(wb.data_ptr()) if wb is not None else None,
                                   ctypes.c_void_p(g.data_ptr()), ctypes.c_void_p(self.m[k].data_ptr()),
                                   ctypes.c_void_p(self.v[k].data_ptr()), lr, beta1, beta2, eps,
                                   weight_decay, self.step_count, self._stream()), "adam")

    # -- data handling
    def standardise(self, feats: np.ndarray):
        x = (np.asarray(feats, np.float32) - self.feat_mean) / self.feat_std
        return self.torch.from_numpy(np.ascontiguousarray(x, np.float32)).to(self.dev)

    def predict(self, feats: np.ndarray) -> np.ndarray:
        """[rows, 2] float64 log-corrections (clipped) for raw feature rows."""
        Y, _ = self.forward(self.standardise(feats))
        out = Y.double().cpu().numpy()
        return np.clip(out, -CLIP, CLIP)

    def save(self, path: str, meta: dict | None = None) -> None:
        os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
        arrs = {f"w{i}": w.cpu().numpy() for i, w in enumerate(self.w)}
        arrs.update({f"b{i}": b.cpu().numpy() for i, b in enumerate(self.b)})
        arrs["feat_mean"] = self.feat_mean
        arrs["feat_std"] = self.feat_std
        arrs["meta"] = np.frombuffer(json.dumps(meta or {}).encode(), np.uint8)
        np.savez_compressed(path, **arrs)

    @classmethod
    def load(cls, path: str, device: int = 0) -> "StageMLP":
        import torch
        d = np.load(path)
        net = cls(device)
        for i in range(len(net.w)):
            net.w[i] = torch.from_numpy(d[f"w{i}"]).to(net.dev)
            net.b[i] = torch.from_numpy(d[f"b{i}"]).to(net.dev)
        net.m = [torch.zeros_like(t) for t in net.w + net.b]
        net.v = [torch.zeros_like(t) for t in net.w + net.b]
        net.feat_mean = d["feat_mean"].astype(np.float32)
        net.feat_std = d["feat_std"].astype(np.float32)
        net._refresh_bf16()
        return net


# ---- proposals -------------------------------------------------------------

def propose_stage_scale(ctx: Context, model: "StageMLP | None", n: int, m: int,
                        raws: np.ndarray) -> np.ndarray:
    """[count, m, 2] (gamma, t) multipliers at equal cost; ones (the plain
    heuristic) where there is no model or a proposal is not finite."""
    raws = np.asarray(raws, np.float64).reshape(len(raws), -1)
    out = np.ones((len(raws), m, 2), np.float32)
    if model is None:
        return out
    feats = np.concatenate([instance_features(n, m, r) for r in raws])
    pred = model.predict(feats).reshape(len(raws), m, 2)
    for k, r in enumerate(raws):
        if not np.all(np.isfinite(pred[k])):
            continue
        g, st, _, _ = schedule(n, m, r)
        _, _, info = ctx.build_diag(n, r)
        sc = equal_cost_scale(n, g, st, float(info.e_abs), pred[k, :, 0], pred[k, :, 1])
        if np.all(np.isfinite(sc)) and np.all(sc > 0):
            out[k] = sc
    return out


def run_with_scale(ctx: Context, n: int, m: int, raws: np.ndarray, scale: np.ndarray | None,
                   samples: int, chunk: int = 64) -> tuple[np.ndarray, int]:
    """Mean P per instance and the total number of Chebyshev terms. Runs in
    plans of `chunk` instances, each executed once (no graph capture)."""
    raws = np.asarray(raws, np.float64).reshape(len(raws), -1)
    ps, terms = [], 0
    for a in range(0, len(raws), chunk):
        sc = None if scale is None else np.ascontiguousarray(scale[a:a + chunk])
        plan = Plan(ctx, n, m, raws[a:a + chunk].ravel(), samples=samples, stage_scale=sc, graph=0)
        plan.execute()
        ps.append(plan.results()["p"])
        terms += plan.stats()["terms"]
        plan.close()
    return np.concatenate(ps), terms


# ---- simulator-generated scans and training --------------------------------

def generate_scans(ctx: Context, count: int, seed: int, n_range=(10, 16), m_range=(2, 5),
                   candidates: int = 16, spread: float = 0.4, samples: int = 20,
                   log=print) -> dict:
    """For `count` seeded SK instances (n, m uniform in the ranges), evaluate
    the heuristic and `candidates` random equal-cost corrections per instance
    with the simulator, and keep the best one's per-stage log-multipliers as
    the targets. Returns feature rows, targets and the scan statistics."""
    rng = np.random.default_rng(seed)
    feats, targets, gains = [], [], []
    t0 = time.time()
    for k in range(count):
        n = int(rng.integers(n_range[0], n_range[1] + 1))
        m = int(rng.integers(m_range[0], m_range[1] + 1))
        raw = sk_instances(n, 1, int(rng.integers(1 << 31)))[0]
        g, st, _, _ = schedule(n, m, raw)
        _, _, info = ctx.build_diag(n, raw)
        cands = [np.zeros((m, 2))] + [rng.uniform(-spread, spread, (m, 2)) for _ in range(candidates)]
        scales = np.stack([equal_cost_scale(n, g, st, float(info.e_abs), c[:, 0], c[:, 1]) for c in cands])
        p, _ = run_with_scale(ctx, n, m, np.tile(raw, (len(cands), 1)), scales, samples)
        best = int(np.argmax(p))
        tgt = np.log(scales[best].astype(np.float64))
        feats.append(instance_features(n, m, raw))
        targets.append(tgt)
        gains.append(p[best] / max(p[0], 1e-12))
        if log and (k + 1) % max(1, count // 10) == 0:
            log(f"scan {k + 1}/{count}  ({time.time() - t0:.1f} s)  mean best/heuristic {np.mean(gains):.4f}")
    return {"features": np.concatenate(feats).astype(np.float32),
            "targets": np.concatenate(targets).astype(np.float32),
            "gain_best_over_heuristic": float(np.mean(gains))}


def train(model: StageMLP, feats: np.ndarray, targets: np.ndarray, steps: int = 3000,
          batch: int = 256, lr: float = 1e-3, seed: int = 0, log=print) -> list[float]:
    torch = model.torch
    model.feat_mean = feats.mean(axis=0).astype(np.float32)
    model.feat_std = (feats.std(axis=0) + 1e-6).astype(np.float32)
    X = model.standardise(feats)
    T = torch.from_numpy(np.ascontiguousarray(targets, np.float32)).to(model.dev)
    rng = np.random.default_rng(seed)
    losses = []
    for s in range(steps):
        idx = torch.from_numpy(rng.integers(0, X.shape[0], batch)).to(model.dev)
        xb, tb = X[idx].contiguous(), T[idx].contiguous()
        Y, acts = model.forward(xb)
        dY = (Y - tb) / batch
        dWs, dbs = model.backward(acts, dY)
        model.adam(dWs, dbs, lr=lr * (0.1 if s > 0.8 * steps else 1.0))
        if s % 100 == 0 or s == steps - 1:
            loss = float(0.5 * ((Y - tb) ** 2).sum().item() / batch)
            losses.append(loss)
            if log and s % 500 == 0:
                log(f"step {s}  loss {loss:.5f}")
    return losses


def evaluate(ctx: Context, model: "StageMLP | None", n: int, m: int, count: int, seed: int,
             samples: int = 100) -> dict:
    """Mean P of the plain heuristic and of the learned proposal (equal cost)
    on `count` fresh seeded SK instances."""
    raws = sk_instances(n, count, seed)
    p_h, terms_h = run_with_scale(ctx, n, m, raws, None, samples)
    scale = propose_stage_scale(ctx, model, n, m, raws)
    p_l, terms_l = run_with_scale(ctx, n, m, raws, scale, samples)
    return {"n": n, "m": m, "instances": count, "samples": samples,
            "mean_p_heuristic": float(p_h.mean()), "mean_p_learned": float(p_l.mean()),
            "ratio": float(p_l.mean() / p_h.mean()),
            "frac_instances_improved": float(np.mean(p_l > p_h)),
            "terms_heuristic": int(terms_h), "terms_learned": int(terms_l)}


def main(argv=None) -> None:
    import argparse
    ap = argparse.ArgumentParser(description="train / evaluate the learned stage schedule")
    ap.add_argument("cmd", choices=["train", "evaluate"])
    ap.add_argument("--out", default=DEFAULT_MODEL)
    ap.add_argument("--scans", type=int, default=5700, help="instances scanned (~20k stage rows)")
    ap.add_argument("--candidates", type=int, default=16)
    ap.add_argument("--scan-samples", type=int, default=20)
    ap.add_argument("--steps", type=int, default=3000)
    ap.add_argument("--eval-count", type=int, default=1024)
    ap.add_argument("--eval-samples", type=int, default=100)
    ap.add_argument("--eval-n", default="18,20")
    ap.add_argument("--seed", type=int, default=2024)
    a = ap.parse_args(argv)
    ctx = Context(0)
    report = {}
    if a.cmd == "train":
        t0 = time.time()
        data = generate_scans(ctx, a.scans, a.seed, candidates=a.candidates, samples=a.scan_samples)
        report["scan"] = {"instances": a.scans, "rows": int(len(data["targets"])),
                          "candidates": a.candidates, "samples": a.scan_samples,
                          "seconds": time.time() - t0,
                          "gain_best_over_heuristic": data["gain_best_over_heuristic"]}
        net = StageMLP(0, seed=a.seed)
        t1 = time.time()
        losses = train(net, data["features"], data["targets"], steps=a.steps, seed=a.seed)
        report["train"] = {"steps": a.steps, "seconds": time.time() - t1,
                           "loss_first": losses[0], "loss_last": losses[-1]}
        net.save(a.out, meta=report)
    net = StageMLP.load(a.out)
    report["evaluate"] = []
    for n in [int(x) for x in a.eval_n.split(",")]:
        r = evaluate(ctx, net, n, 4, a.eval_count, 7000 + n, a.eval_samples)
        report["evaluate"].append(r)
        print(json.dumps(r), flush=True)
    with open(os.path.splitext(a.out)[0] + ".json", "w") as f:
        json.dump(report, f, indent=1)
    print(json.dumps(report), flush=True)


if __name__ == "__main__":
    main()
