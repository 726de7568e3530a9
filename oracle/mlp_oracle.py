"""ORACLE — test infrastructure only: float64 numpy restatement of the learned
schedule's MLP layers (the CUDA kernels in multistageqw_b200/csrc/mqw_mlp.cu)
for gradient checks. Weights are rounded to bfloat16 exactly as the product
stores them (round to nearest, ties to even); everything else is float64.

The MLP has no counterpart in the reference, so there is nothing of the
reference to pin it to; its own pin is the finite-difference check in
tests/test_learned.py.
"""
from __future__ import annotations

import numpy as np


def bf16_round(x: np.ndarray) -> np.ndarray:
    """float32 -> nearest bfloat16 (ties to even), returned as float32."""
    x = np.ascontiguousarray(x, dtype=np.float32)
    b = x.view(np.uint32).astype(np.uint64)
    bias = 0x7FFF + ((b >> 16) & 1)
    r = ((b + bias) & 0xFFFF0000).astype(np.uint32)
    return r.view(np.float32)


def linear_forward(X, W, b, relu):
    """Y = X W^T + b (ReLU optional), W rounded to bfloat16."""
    Wb = bf16_round(W).astype(np.float64)
    Z = X.astype(np.float64) @ Wb.T
    if b is not None:
        Z = Z + b.astype(np.float64)
    return np.maximum(Z, 0.0) if relu else Z


def linear_backward(X, W, Y, dY, relu):
    """(dX, dW, db) for Y = act(X W^T + b) with bfloat16-rounded W."""
    Wb = bf16_round(W).astype(np.float64)
    dZ = dY.astype(np.float64) * ((Y > 0) if relu else 1.0)
    dW = dZ.T @ X.astype(np.float64)
    db = dZ.sum(axis=0)
    dX = dZ @ Wb
    return dX, dW, db


def mlp_forward(params, X):
    """params: list of (W, b); ReLU on every layer but the last. Returns the
    output and the per-layer activations (input first)."""
    acts = [np.asarray(X, np.float64)]
    for li, (W, b) in enumerate(params):
        relu = li < len(params) - 1
        acts.append(linear_forward(acts[-1], W, b, relu))
    return acts[-1], acts


def mlp_loss_grad(params, X, T):
    """Mean squared error 0.5*mean(sum((Y - T)^2)) and its gradients."""
    Y, acts = mlp_forward(params, X)
    B = X.shape[0]
    loss = 0.5 * np.sum((Y - T) ** 2) / B
    d = (Y - T) / B
    grads = [None] * len(params)
    for li in range(len(params) - 1, -1, -1):
        W, b = params[li]
        relu = li < len(params) - 1
        dX, dW, db = linear_backward(acts[li], W, acts[li + 1], d, relu)
        grads[li] = (dW, db)
        d = dX
    return loss, grads
