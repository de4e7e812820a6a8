"""Collision-likelihood surrogate: a bank of BF16 MLPs (one per plant) run by
the library's tensor-core kernels (csd_mlp_*).

Each net maps a configuration q (scaled by 1/pi, zero padded to 16) through
three ReLU layers of width 256 to one logit, P(collision) = sigmoid(logit).
It is trained on configurations labelled by the exact checker and only ever
orders work: every verdict is still the exact checker's.
"""
from __future__ import annotations

import ctypes
import math
from typing import Optional, Sequence, Tuple

import numpy as np

from . import _capi as C


def num_params() -> int:
    return int(C.lib().csd_mlp_num_params())


class CollisionSurrogate:
    """`dims[i]` is the input dimension (plant DOF) of net i."""

    def __init__(self, dims: Sequence[int], seed: int = 0, in_scale: float = 1.0 / math.pi):
        self.dims = [int(d) for d in dims]
        arr = np.ascontiguousarray(np.asarray(self.dims, np.int32))
        h = ctypes.c_void_p()
        C.check(C.lib().csd_mlp_create(len(self.dims), C.ptr(arr), ctypes.c_float(in_scale), ctypes.c_uint64(seed),
                                       ctypes.byref(h)))
        self._handle = h
        self.P = num_params()

    @property
    def handle(self) -> ctypes.c_void_p:
        return self._handle

    @property
    def nets(self) -> int:
        return len(self.dims)

    def params(self) -> np.ndarray:
        out = np.zeros((self.nets, self.P), np.float32)
        C.check(C.lib().csd_mlp_get_params(self._handle, C.ptr(out)))
        return out

    def set_params(self, params: np.ndarray) -> None:
        p = np.ascontiguousarray(np.asarray(params, np.float32).reshape(self.nets, self.P))
        C.check(C.lib().csd_mlp_set_params(self._handle, C.ptr(p)))

    def logits(self, blocks: Sequence[Tuple[int, np.ndarray]]) -> list:
        """blocks: (net index, configurations [rows, dim]) -> logits per block."""
        nets = np.asarray([b[0] for b in blocks], np.int32)
        rows = np.asarray([len(b[1]) for b in blocks], np.int32)
        for n, x in blocks:
            if np.asarray(x).ndim != 2 or np.asarray(x).shape[1] != self.dims[n]:
                raise ValueError("configurations must be [rows, dim] with the net's dimension")
        x = np.ascontiguousarray(np.concatenate([np.asarray(b[1], np.float32).reshape(-1) for b in blocks]))
        out = np.zeros(int(rows.sum()), np.float32)
        C.check(C.lib().csd_mlp_infer(self._handle, len(blocks), C.ptr(nets), C.ptr(rows), C.ptr(x), C.ptr(out),
                                      C.CSD_PTR_HOST, None))
        res, o = [], 0
        for r in rows:
            res.append(out[o:o + r].copy())
            o += r
        return res

    def gradients(self, x: Sequence[np.ndarray], y: Sequence[np.ndarray]):
        """One forward + backward pass: x[i] [batch, dims[i]], y[i] [batch] in
        {0, 1} -> (gradients [nets, P], mean BCE loss [nets])."""
        batch = len(x[0])
        xs = np.ascontiguousarray(np.concatenate([np.asarray(a, np.float32).reshape(-1) for a in x]))
        ys = np.ascontiguousarray(np.concatenate([np.asarray(b, np.uint8).reshape(-1) for b in y]))
        g = np.zeros((self.nets, self.P), np.float32)
        loss = np.zeros(self.nets, np.float32)
        C.check(C.lib().csd_mlp_gradients(self._handle, C.ptr(xs), C.ptr(ys), batch, C.ptr(g), C.ptr(loss)))
        return g, loss

    def train(self, x: Sequence[np.ndarray], y: Sequence[np.ndarray], batch: int = 512, epochs: float = 4.0,
              lr: float = 1e-3, seed: int = 0) -> np.ndarray:
        """Adam on every net at once: x[i] [n, dims[i]] configurations, y[i] [n]
        exact verdicts (1 = colliding). n is cut to a multiple of batch; rows
        are shuffled once. Returns the mean loss of every step."""
        import torch
        n = min(len(a) for a in x)
        n -= n % batch
        if n < batch:
            raise ValueError("need at least one batch of data per net")
        rng = np.random.default_rng(seed)
        xs, ys = [], []
        for a, b in zip(x, y):
            perm = rng.permutation(len(a))[:n]
            xs.append(np.asarray(a, np.float32)[perm].reshape(-1))
            ys.append(np.asarray(b, np.uint8)[perm])
        tx = torch.from_numpy(np.concatenate(xs)).cuda()
        ty = torch.from_numpy(np.concatenate(ys)).cuda()
        steps = int(round(epochs * n / batch))
        hist = np.zeros(max(steps, 1), np.float32)
        C.check(C.lib().csd_mlp_train(self._handle, C.ptr(tx.data_ptr()), C.ptr(ty.data_ptr()), n, batch, steps,
                                      ctypes.c_float(lr), C.ptr(hist), None))
        return hist[:steps]

    def __del__(self):
        h = getattr(self, "_handle", None)
        if h and C is not None and C._lib is not None:
            try:
                C._lib.csd_mlp_destroy(h)
            except Exception:  # pragma: no cover
                pass
        self._handle = None


def gemm_test(a_bits: np.ndarray, b_bits: np.ndarray) -> np.ndarray:
    """D = A B^T through the tensor-core GEMM; A [M, K], B [N, K] as bf16 bit
    patterns (uint16), N 16 or 256."""
    a = np.ascontiguousarray(a_bits, np.uint16)
    b = np.ascontiguousarray(b_bits, np.uint16)
    M, K = a.shape
    N = b.shape[0]
    d = np.zeros((M, N), np.float32)
    C.check(C.lib().csd_mlp_gemm_test(C.ptr(a), C.ptr(b), M, N, K, C.ptr(d)))
    return d


def training_set(scene, seed_edges, n: int, seed: int, sigma: float = 0.35, local_fraction: float = 0.5):
    """n configurations of `scene` labelled by the exact checker (1 =
    colliding): (1 - local_fraction) uniform in the joint limits, the rest
    around the seed edges (a uniform point of a random edge plus N(0, sigma^2)
    per joint, clipped to the limits). Returns (x [n, dim] f32, y [n] u8)."""
    from .api import CheckCollisionFreeCuda
    rng = np.random.default_rng(seed)
    lo, hi = scene.lower(), scene.upper()
    n_loc = int(round(n * local_fraction)) if seed_edges else 0
    x = np.empty((n, scene.dim), np.float32)
    x[:n - n_loc] = lo + (hi - lo) * rng.random((n - n_loc, scene.dim))
    if n_loc:
        e = rng.integers(0, len(seed_edges), n_loc)
        t = rng.random(n_loc)[:, None]
        a = np.stack([seed_edges[i][0] for i in e])
        b = np.stack([seed_edges[i][1] for i in e])
        x[n - n_loc:] = np.clip(a + t * (b - a) + rng.normal(0, sigma, (n_loc, scene.dim)), lo, hi)
    y = (CheckCollisionFreeCuda(x.T, scene.plant) == 0).astype(np.uint8)
    return x, y
