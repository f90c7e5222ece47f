"""CPU restatement of the order-selection MLP (FP64 numpy).  TEST INFRASTRUCTURE.

The network has no counterpart in the reference (which picks one order from
eps by a fixed formula, cpu/multipole3d.cpp:1328-1331); this module is the
checker for the CUDA forward / backward / Adam kernels in
``laplace_fmm_b200/csrc/mlp.cu``: same parameter layout, same masked
mean-squared-error loss, same Adam update with bias correction.

Layout (floats): W1[64][16] b1[64] W2[64][64] b2[64] W3[14][64] b3[14].
"""
from __future__ import annotations

import numpy as np

F, H, O = 16, 64, 14
SHAPES = [("W1", (H, F)), ("b1", (H,)), ("W2", (H, H)), ("b2", (H,)), ("W3", (O, H)), ("b3", (O,))]
NPARAM = sum(int(np.prod(s)) for _, s in SHAPES)


def unpack(params):
    out, off = {}, 0
    for name, shape in SHAPES:
        n = int(np.prod(shape))
        out[name] = np.asarray(params[off:off + n], dtype=np.float64).reshape(shape)
        off += n
    return out


def pack(parts):
    return np.concatenate([np.asarray(parts[name], dtype=np.float64).ravel() for name, _ in SHAPES])


def init(seed=0):
    """He-uniform weights, zero biases (the trainer's initialisation)."""
    rng = np.random.default_rng(seed)
    parts = {}
    for name, shape in SHAPES:
        if name.startswith("W"):
            bound = np.sqrt(6.0 / shape[1])
            parts[name] = rng.uniform(-bound, bound, size=shape)
        else:
            parts[name] = np.zeros(shape)
    return pack(parts).astype(np.float32)


def forward(params, X, keep=False):
    p = unpack(params)
    X = np.asarray(X, dtype=np.float64)
    A1 = np.maximum(X @ p["W1"].T + p["b1"], 0.0)
    A2 = np.maximum(A1 @ p["W2"].T + p["b2"], 0.0)
    Y = A2 @ p["W3"].T + p["b3"]
    return (Y, A1, A2) if keep else Y


def loss_and_grad(params, X, T, M):
    """L = sum M (Y - T)^2 / sum M and dL/dparams (packed)."""
    p = unpack(params)
    X = np.asarray(X, dtype=np.float64)
    T = np.asarray(T, dtype=np.float64)
    M = np.asarray(M, dtype=np.float64)
    Y, A1, A2 = forward(params, X, keep=True)
    cnt = M.sum() if M.sum() > 0 else 1.0
    E = Y - T
    loss = float((M * E * E).sum() / cnt)
    D3 = 2.0 * M * E / cnt
    D2 = (D3 @ p["W3"]) * (A2 > 0)
    D1 = (D2 @ p["W2"]) * (A1 > 0)
    g = {"W3": D3.T @ A2, "b3": D3.sum(0), "W2": D2.T @ A1, "b2": D2.sum(0), "W1": D1.T @ X, "b1": D1.sum(0)}
    return loss, pack(g)


def adam(params, grad, m, v, step, lr=1e-3, beta1=0.9, beta2=0.999, eps=1e-8):
    """One Adam step; returns (params, m, v)."""
    m = beta1 * m + (1 - beta1) * grad
    v = beta2 * v + (1 - beta2) * grad * grad
    c1 = 1 - beta1 ** step
    c2 = 1 - beta2 ** step
    return params - lr * (m / c1) / (np.sqrt(v / c2) + eps), m, v
