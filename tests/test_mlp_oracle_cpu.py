"""The CPU restatement of the rank model (oracle/mlp.py) against finite
differences of its own loss, and its BF16 rounding against hand-checked bit
patterns.  The library's kernels are checked against this restatement on
the GPU (tests/test_mlp_gpu.py)."""
import numpy as np

from oracle import mlp as om


def test_bf16_rounding_bits():
    # BF16 keeps 8 significant bits: near 1 the spacing is 2^-7.  1 + 2^-7 is
    # exact; 1 + 2^-8 is a tie that rounds to even (1.0); 1 + 3 * 2^-8 is a
    # tie that rounds to even (1 + 2^-6); 1 + 3 * 2^-10 rounds down; -3.140625
    # (binary 11.001001) is exact
    x = np.array([1.0, 1.0078125, 1.00390625, 1.01171875, 1.0029296875, -3.140625, 0.0], dtype=np.float32)
    want = np.array([1.0, 1.0078125, 1.0, 1.015625, 1.0, -3.140625, 0.0], dtype=np.float32)
    assert np.array_equal(om.bf16_round(x), want)


def test_gradient_matches_finite_differences():
    rng = np.random.default_rng(3)
    p = rng.standard_normal(om.NP) * 0.3
    X = rng.standard_normal((40, om.IN))
    t = rng.standard_normal(40)
    mean, scale = rng.standard_normal(om.IN) * 0.1, 1.0 + rng.random(om.IN)
    loss, g = om.loss_and_grad(p, X, t, mean, scale)
    h = 1e-6
    for q in rng.choice(om.NP, 60, replace=False):
        e = np.zeros(om.NP)
        e[q] = h
        lp, _ = om.loss_and_grad(p + e, X, t, mean, scale)
        lm, _ = om.loss_and_grad(p - e, X, t, mean, scale)
        fd = (lp - lm) / (2 * h)
        assert abs(fd - g[q]) <= 1e-6 * max(1.0, abs(g[q])), (q, fd, g[q])
    assert loss > 0
