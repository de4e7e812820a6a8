"""Surrogate MLP on the tensor cores: the tcgen05 GEMM against numpy, the
fused forward and the backward pass against the CPU oracle (bf16 rounding at
the same points), and training."""
import math

import numpy as np
import pytest

from csdecomp_b200 import surrogate as S
from oracle import mlp_oracle as M

pytestmark = pytest.mark.gpu


def bf16_bits(x):
    f = np.ascontiguousarray(np.asarray(x, np.float32))
    u = f.view(np.uint32).astype(np.uint64)
    return (((u + 0x7FFF + ((u >> 16) & 1)) >> 16) & 0xFFFF).astype(np.uint16)


def bits_to_f64(b):
    return (b.astype(np.uint32) << 16).view(np.float32).astype(np.float64)


@pytest.mark.parametrize("M_, N, K", [(128, 256, 64), (300, 256, 136), (256, 16, 512), (77, 16, 24)])
def test_gemm_matches_numpy(M_, N, K):
    rng = np.random.default_rng(M_ + N + K)
    a = bf16_bits(rng.normal(size=(M_, K)))
    b = bf16_bits(rng.normal(size=(N, K)))
    d = S.gemm_test(a, b)
    ref = bits_to_f64(a) @ bits_to_f64(b).T
    err = np.abs(d - ref).max() / np.abs(ref).max()
    assert err < 1e-5, err


def make_net(dims, seed=3):
    net = S.CollisionSurrogate(dims, seed=seed)
    # make biases non-zero so that they are exercised
    p = net.params()
    rng = np.random.default_rng(seed)
    for s, e in [(M.oB1, M.oW2), (M.oB2, M.oW3), (M.oB3, M.oW4)]:
        p[:, s:e] = rng.normal(0, 0.05, (p.shape[0], e - s))
    p[:, M.oB4] = 0.2
    net.set_params(p)
    return net, net.params()


def test_forward_matches_oracle():
    dims = [7, 14]
    net, p = make_net(dims)
    rng = np.random.default_rng(1)
    xs = [rng.uniform(-math.pi, math.pi, (300, 7)), rng.uniform(-math.pi, math.pi, (129, 14))]
    got = net.logits([(0, xs[0]), (1, xs[1])])
    for i in range(2):
        ref, _ = M.forward(p[i].astype(np.float64), xs[i], 1 / math.pi)
        err = np.abs(got[i] - ref) / (1 + np.abs(ref))
        assert np.quantile(err, 0.99) < 1e-2 and err.max() < 5e-2, (i, err.max())


def test_gradients_match_oracle():
    dims = [7, 14]
    net, p = make_net(dims, seed=5)
    rng = np.random.default_rng(2)
    B = 128
    xs = [rng.uniform(-math.pi, math.pi, (B, d)) for d in dims]
    ys = [rng.integers(0, 2, B).astype(np.uint8) for _ in dims]
    g, loss = net.gradients(xs, ys)
    blocks = [(M.oW1, M.oB1), (M.oB1, M.oW2), (M.oW2, M.oB2), (M.oB2, M.oW3), (M.oW3, M.oB3), (M.oB3, M.oW4),
              (M.oW4, M.oB4), (M.oB4, M.P)]
    for i in range(len(dims)):
        lref, gref = M.loss_and_grad(p[i].astype(np.float64), xs[i], ys[i], 1 / math.pi)
        assert abs(loss[i] - lref) < 1e-3 * max(1.0, lref)
        for s, e in blocks:
            num = np.linalg.norm(g[i, s:e] - gref[s:e])
            den = np.linalg.norm(gref[s:e]) + 1e-12
            assert num / den < 2e-2, (i, s, e, num / den)


def test_training_learns_a_ball():
    """Label = configuration inside a ball; a few epochs fit it."""
    dims = [7]
    net = S.CollisionSurrogate(dims, seed=9)
    rng = np.random.default_rng(4)
    x = rng.uniform(-math.pi, math.pi, (16384, 7)).astype(np.float32)
    y = (np.linalg.norm(x - 0.5, axis=1) < 3.5).astype(np.uint8)
    hist = net.train([x], [y], batch=512, epochs=6, lr=2e-3)
    assert hist[-8:].mean() < 0.5 * hist[:8].mean()
    xt = rng.uniform(-math.pi, math.pi, (4096, 7)).astype(np.float32)
    yt = np.linalg.norm(xt - 0.5, axis=1) < 3.5
    pred = net.logits([(0, xt)])[0] > 0
    assert (pred == yt).mean() > 0.9
