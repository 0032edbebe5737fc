"""CPU restatement of the library's rank model -- TEST INFRASTRUCTURE ONLY.

The 6 -> 64 -> 64 -> 1 perceptron (ReLU) of rcs_b200/csrc/mlp.cu in float64
numpy, with the library's conventions: the weights used by the forward and
backward passes are the BF16 rounding (round to nearest, ties to even) of
the FP32 master weights; inputs are normalised as (x - mean) * scale; the loss
is the mean squared error (1/n) sum (y_i - t_i)^2.  The model has no
counterpart in the reference (vaishna77/RCS), so this restatement is pinned
against finite differences of itself (tests/test_mlp_oracle_cpu.py) and the
library's kernels against it.

Parameter layout (4,673 floats): W1 [64 x 6] row-major, b1 [64], W2 [64 x 64]
row-major (output, input), b2 [64], w3 [64], b3.
"""
from __future__ import annotations

import numpy as np

IN, H = 6, 64
W1, B1 = 0, H * IN
W2 = B1 + H
B2 = W2 + H * H
W3 = B2 + H
B3 = W3 + H
NP = B3 + 1


def bf16_round(x) -> np.ndarray:
    """FP32 -> nearest BF16 (ties to even), returned as float32."""
    b = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    b = (b + 0x7FFF + ((b >> 16) & 1)) & 0xFFFF0000
    return b.astype(np.uint32).view(np.float32)


def unpack(p):
    p = np.asarray(p, dtype=np.float64)
    return (p[W1:B1].reshape(H, IN), p[B1:W2], p[W2:B2].reshape(H, H), p[B2:W3], p[W3:B3], p[B3])


def forward(p, X, mean, scale):
    """Outputs y (n) and the intermediates of the backward pass."""
    w1, b1, w2, b2, w3, b3 = unpack(p)
    x = (np.asarray(X, np.float64) - np.asarray(mean, np.float64)) * np.asarray(scale, np.float64)
    z1 = x @ w1.T + b1
    a1 = np.maximum(z1, 0.0)
    z2 = a1 @ w2.T + b2
    a2 = np.maximum(z2, 0.0)
    y = a2 @ w3 + b3
    return y, (x, z1, a1, z2, a2)


def loss_and_grad(p, X, t, mean, scale):
    """(loss, gradient) of the mean squared error at parameters p."""
    w1, b1, w2, b2, w3, b3 = unpack(p)
    y, (x, z1, a1, z2, a2) = forward(p, X, mean, scale)
    n = len(y)
    r = y - np.asarray(t, np.float64)
    dy = 2.0 * r / n
    g = np.zeros(NP)
    g[W3:B3] = a2.T @ dy
    g[B3] = dy.sum()
    d2 = np.outer(dy, w3) * (z2 > 0)
    g[W2:B2] = (d2.T @ a1).ravel()
    g[B2:W3] = d2.sum(axis=0)
    d1 = (d2 @ w2) * (z1 > 0)
    g[W1:B1] = (d1.T @ x).ravel()
    g[B1:W2] = d1.sum(axis=0)
    return float(np.mean(r * r)), g


def library_grad(master, X, t, mean, scale):
    """What aifmm_mlp_grad computes: the gradient at the BF16-rounded master weights."""
    return loss_and_grad(bf16_round(master).astype(np.float64), X, t, mean, scale)
