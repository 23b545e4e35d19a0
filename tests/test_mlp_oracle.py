"""The MLP oracle (CPU): its backward pass agrees with central finite
differences of its own loss when BF16 rounding is off, and its BF16 rounding
is round-to-nearest-even."""
import os
import sys

import numpy as np

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
import mlp_oracle as mo  # noqa: E402


def test_bf16_rounding():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, -2.5, 3.14159265], np.float32)
    b = mo.bf16(x)
    assert b[0] == 1.0
    assert b[1] == 1.0  # tie -> even
    assert b[2] == 1.0 + 4 * 2 ** -8  # tie -> even (upwards)
    assert b[3] == -2.5
    assert abs(b[4] - 3.140625) < 1e-12


def test_gradients_match_finite_differences():
    rng = np.random.default_rng(0)
    dims = [6, 10, 8, 5]
    n = sum(dims[l] * dims[l + 1] + dims[l + 1] for l in range(len(dims) - 1))
    p = rng.normal(0, 0.5, n)
    X = rng.normal(0, 1, (7, dims[0]))
    T = np.concatenate([rng.normal(0, 1, (7, dims[-1] - 1)), (rng.random((7, 1)) > 0.5)], 1).astype(np.float64)
    loss, g = mo.loss_and_grad(p, dims, X, T, rounding=False)
    eps = 1e-6
    for i in rng.choice(n, 40, replace=False):
        q = p.copy()
        q[i] += eps
        lp, _ = mo.loss_and_grad(q, dims, X, T, rounding=False)
        q[i] -= 2 * eps
        lm, _ = mo.loss_and_grad(q, dims, X, T, rounding=False)
        fd = (lp - lm) / (2 * eps)
        assert abs(fd - g[i]) < 1e-6 + 1e-5 * abs(fd), (i, fd, g[i])
