"""NumPy oracle of the correction MLP -- TEST INFRASTRUCTURE.

Restates the forward pass and the backward pass of the BF16 tensor-core
kernels (n-body-2d_b200/csrc/k_mlp.cu) in FP64, rounding to BF16 exactly where
the kernels round: inputs, weights and hidden activations enter the matrix
products as BF16; the gradients entering the backward products (dy, dp2, dp1)
are BF16; accumulations are exact here (FP32 on the GPU).  exact=True drops all
rounding, for a finite-difference check of the backward pass itself.
"""
from __future__ import annotations

import numpy as np

H, NIN = 64, 12
W1, B1 = 0, H * NIN
W2 = B1 + H
B2 = W2 + H * H
W3 = B2 + H
B3 = W3 + 2 * H
YS = B3 + 2
PARAMS = YS + 1


def bf16(x) -> np.ndarray:
    """Round to the nearest BF16 (ties to even), returned as float64."""
    f = np.ascontiguousarray(x, dtype=np.float32)
    b = f.view(np.uint32).astype(np.uint64)
    b = (b + 0x7FFF + ((b >> 16) & 1)) & 0xFFFF0000
    return b.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(p):
    p = np.asarray(p, dtype=np.float64)
    return (p[W1:B1].reshape(H, NIN), p[B1:W2], p[W2:B2].reshape(H, H), p[B2:W3],
            p[W3:B3].reshape(2, H), p[B3:YS], p[YS])


def forward(p, X, exact=False):
    r = (lambda v: np.asarray(v, dtype=np.float64)) if exact else bf16
    w1, b1, w2, b2, w3, b3, _ = unpack(p)
    x = r(X)
    h1 = r(np.tanh(x @ r(w1).T + b1))
    h2 = r(np.tanh(h1 @ r(w2).T + b2))
    y = h2 @ r(w3).T + b3
    return y, (x, h1, h2)


def loss_grad(p, X, T, exact=False):
    """Mean over samples of |y - t|^2 and its gradient (layout of the ABI)."""
    r = (lambda v: np.asarray(v, dtype=np.float64)) if exact else bf16
    w1, b1, w2, b2, w3, b3, _ = unpack(p)
    y, (x, h1, h2) = forward(p, X, exact)
    n = X.shape[0]
    d = y - np.asarray(T, dtype=np.float64)
    loss = float((d * d).sum() / n)
    dy = 2.0 * d / n
    dp2 = (r(dy) @ r(w3)) * (1.0 - h2 * h2)
    dp1 = (r(dp2) @ r(w2)) * (1.0 - h1 * h1)
    g = np.zeros(PARAMS)
    g[W3:B3] = (r(dy).T @ h2).ravel()
    g[B3:YS] = dy.sum(0)
    g[W2:B2] = (r(dp2).T @ h1).ravel()
    g[B2:W3] = dp2.sum(0)
    g[W1:B1] = (r(dp1).T @ x).ravel()
    g[B1:W2] = dp1.sum(0)
    return loss, g


def init(seed: int = 0) -> np.ndarray:
    rng = np.random.default_rng(seed)
    p = np.zeros(PARAMS)
    p[W1:B1] = rng.uniform(-1, 1, H * NIN) * np.sqrt(6.0 / (NIN + H))
    p[W2:B2] = rng.uniform(-1, 1, H * H) * np.sqrt(6.0 / (2 * H))
    p[W3:B3] = rng.uniform(-1, 1, 2 * H) * np.sqrt(6.0 / (H + 2))
    p[B1:W2] = rng.normal(0, 0.1, H)
    p[B2:W3] = rng.normal(0, 0.1, H)
    p[B3:YS] = rng.normal(0, 0.1, 2)
    p[YS] = 1.0
    return p
