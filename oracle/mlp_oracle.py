"""CPU oracle of the surrogate MLP (test infrastructure only).

Forward and backward of in -> 256 -> 256 -> 256 -> 1 with ReLU and mean
binary cross-entropy with logits, in float64, rounding to bfloat16 exactly
where the tensor-core kernels store bf16: the scaled input, W1..W3, the
hidden activations H1..H3 and the back-propagated dZ3..dZ1. Products of
bf16 values are exact in float64, so the only differences left against the
GPU are its float32 accumulation order and the rare bf16 rounding that this
flips. Parameter layout per net: W1 [256][16], b1, W2 [256][256], b2, W3, b3,
w4 [256], b4 (row-major [out][in]).

The backward pass is checked against central finite differences of the
float64 forward without rounding (tests/test_oracle_mlp.py).
"""
from __future__ import annotations

import numpy as np

H, IN = 256, 16
oW1 = 0
oB1 = oW1 + H * IN
oW2 = oB1 + H
oB2 = oW2 + H * H
oW3 = oB2 + H
oB3 = oW3 + H * H
oW4 = oB3 + H
oB4 = oW4 + H
P = oB4 + 1


def bf16(x) -> np.ndarray:
    """Round to bfloat16 (nearest, ties to even) and return as float64."""
    f = np.ascontiguousarray(np.asarray(x, np.float32))
    u = f.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    r = np.where(np.isnan(f), u, r)
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(p: np.ndarray):
    p = np.asarray(p, np.float64)
    return (p[oW1:oB1].reshape(H, IN), p[oB1:oW2], p[oW2:oB2].reshape(H, H), p[oB2:oW3],
            p[oW3:oB3].reshape(H, H), p[oB3:oW4], p[oW4:oB4], p[oB4])


def pad_input(x: np.ndarray, scale: float) -> np.ndarray:
    x = np.asarray(x, np.float32) * np.float32(scale)
    out = np.zeros((len(x), IN), np.float32)
    out[:, :x.shape[1]] = x
    return out


def forward(p, x, scale, rounding=True):
    """Returns (logits, cache) for x [B, dim]."""
    W1, b1, W2, b2, W3, b3, w4, b4 = unpack(p)
    rd = bf16 if rounding else (lambda a: np.asarray(a, np.float64))
    X = rd(pad_input(x, scale))
    W1r, W2r, W3r = rd(W1), rd(W2), rd(W3)
    Z1 = X @ W1r.T + b1
    H1 = rd(np.maximum(Z1, 0))
    Z2 = H1 @ W2r.T + b2
    H2 = rd(np.maximum(Z2, 0))
    Z3 = H2 @ W3r.T + b3
    H3 = rd(np.maximum(Z3, 0))
    z = H3 @ w4 + b4
    return z, (X, H1, H2, H3, W2r, W3r)


def loss_and_grad(p, x, y, scale, rounding=True):
    """Mean BCE-with-logits loss and its gradient [P] (float64)."""
    W1, b1, W2, b2, W3, b3, w4, b4 = unpack(p)
    rd = bf16 if rounding else (lambda a: np.asarray(a, np.float64))
    z, (X, H1, H2, H3, W2r, W3r) = forward(p, x, scale, rounding)
    y = np.asarray(y, np.float64)
    B = len(z)
    loss = np.mean(np.maximum(z, 0) - z * y + np.log1p(np.exp(-np.abs(z))))
    dz = (1.0 / (1.0 + np.exp(-z)) - y) / B
    g = np.zeros(P)
    g[oW4:oB4] = H3.T @ dz
    g[oB4] = dz.sum()
    dZ3 = rd(np.outer(dz, w4) * (H3 > 0))
    g[oW3:oB3] = (dZ3.T @ H2).reshape(-1)
    g[oB3:oW4] = dZ3.sum(0)
    dZ2 = rd((dZ3 @ W3r) * (H2 > 0))
    g[oW2:oB2] = (dZ2.T @ H1).reshape(-1)
    g[oB2:oW3] = dZ2.sum(0)
    dZ1 = rd((dZ2 @ W2r) * (H1 > 0))
    g[oW1:oB1] = (dZ1.T @ X).reshape(-1)
    g[oB1:oW2] = dZ1.sum(0)
    return loss, g
