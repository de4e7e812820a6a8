"""Pins the surrogate MLP oracle: its backward pass against central finite
differences of its own float64 forward (no bf16 rounding)."""
import math

import numpy as np

from oracle import mlp_oracle as M


def small_params(rng):
    p = np.zeros(M.P)
    p[M.oW1:M.oB1] = rng.normal(0, 0.5, M.H * M.IN)
    p[M.oB1:M.oW2] = rng.normal(0, 0.1, M.H)
    p[M.oW2:M.oB2] = rng.normal(0, 1 / 16, M.H * M.H)
    p[M.oB2:M.oW3] = rng.normal(0, 0.1, M.H)
    p[M.oW3:M.oB3] = rng.normal(0, 1 / 16, M.H * M.H)
    p[M.oB3:M.oW4] = rng.normal(0, 0.1, M.H)
    p[M.oW4:M.oB4] = rng.normal(0, 0.1, M.H)
    p[M.oB4] = 0.1
    return p


def test_backward_matches_finite_differences():
    rng = np.random.default_rng(0)
    p = small_params(rng)
    x = rng.uniform(-math.pi, math.pi, (24, 7))
    y = rng.integers(0, 2, 24)
    _, g = M.loss_and_grad(p, x, y, 1 / math.pi, rounding=False)
    idx = np.concatenate([rng.choice(np.arange(s, e), 6, replace=False)
                          for s, e in [(M.oW1, M.oB1), (M.oB1, M.oW2), (M.oW2, M.oB2), (M.oB2, M.oW3),
                                       (M.oW3, M.oB3), (M.oB3, M.oW4), (M.oW4, M.oB4)]] + [[M.oB4]])
    eps = 1e-6
    for i in idx:
        q = p.copy()
        q[i] += eps
        lp, _ = M.loss_and_grad(q, x, y, 1 / math.pi, rounding=False)
        q[i] -= 2 * eps
        lm, _ = M.loss_and_grad(q, x, y, 1 / math.pi, rounding=False)
        fd = (lp - lm) / (2 * eps)
        assert abs(fd - g[i]) <= 1e-6 + 1e-4 * abs(fd), (i, fd, g[i])


def test_bf16_rounding():
    # bf16 spacing at 1 is 2^-7
    v = np.array([1.0078125, 1.00390625, 1.01171875, 1.005, -3.3, 0.0], np.float32)
    r = M.bf16(v)
    assert r[0] == 1.0078125    # representable: kept
    assert r[1] == 1.0          # halfway, ties to the even mantissa (down)
    assert r[2] == 1.015625     # halfway, ties to the even mantissa (up)
    assert r[3] == 1.0078125    # nearest
    assert r[4] == -3.296875
    assert r[5] == 0.0
