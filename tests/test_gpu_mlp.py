"""Surrogate MLP on the tensor cores (tcgen05, BF16 x BF16 -> FP32 in TMEM)
against the CPU oracle (oracle/mlp_oracle.py).

* GEMM: c = a . b^T (+ bias, ReLU) for the shapes the MLP uses, ragged row
  counts included; |c - ref| <= 2e-5 * sum_k |a_ik b_jk| + 1e-6 (FP32
  accumulation of BF16 products; the reference sums in float64).
* gradients of one batch: per-layer relative L2 error < 1e-2 (BF16 rounding
  of an intermediate may flip where FP32 and float64 sums differ in the last
  bit), loss within 1e-3 relative.
* inference: relative L2 error of the outputs < 1e-2.
* training: the loss on a smooth synthetic target falls by 5x.
"""
import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
import mlp_oracle as mo  # noqa: E402

pytestmark = pytest.mark.gpu

DIMS = [32, 256, 256, 256, 59]


@pytest.mark.parametrize("m,n,k", [(256, 256, 256), (300, 64, 256), (128, 32, 256), (77, 256, 32), (512, 16, 16)])
def test_gemm_matches_float64(built, m, n, k):
    rng = np.random.default_rng(m * 7 + n + k)
    a = rng.normal(0, 1, (m, k)).astype(np.float32)
    b = rng.normal(0, 1, (n, k)).astype(np.float32)
    bias = rng.normal(0, 1, n).astype(np.float32)
    ab, bb = mo.bf16_bits(a), mo.bf16_bits(b)
    af, bf = mo.bf16(a), mo.bf16(b)
    for relu, bs in ((False, None), (True, bias)):
        c = built.mlp_gemm(ab, bb, bias=bs, relu=relu).astype(np.float64)
        ref = af @ bf.T + (0 if bs is None else bs.astype(np.float64))
        if relu:
            ref = np.maximum(ref, 0)
        scale = np.abs(af) @ np.abs(bf).T + (0 if bs is None else np.abs(bs))
        err = np.abs(c - ref)
        assert np.all(err <= 2e-5 * scale + 1e-6), err.max()


def _data(rng, rows):
    x = rng.uniform(-1, 1, (rows, DIMS[0])).astype(np.float32)
    nr = DIMS[-1] - 1
    # a smooth target: log-rates from a fixed random two-layer map, label from their mean
    w1 = np.random.default_rng(99).normal(0, 0.4, (DIMS[0], 64))
    w2 = np.random.default_rng(98).normal(0, 0.3, (64, nr))
    lr_ = np.log1p(np.exp(np.tanh(x @ w1) @ w2 + 1.5))
    lab = (lr_.mean(1) > np.median(lr_.mean(1))).astype(np.float32)
    return x, np.concatenate([lr_, lab[:, None]], 1).astype(np.float32)


def test_gradients_match_oracle(built):
    rng = np.random.default_rng(1)
    net = built.Mlp(DIMS, seed=5)
    try:
        p = net.get_params()
        assert p.size == net.param_count()
        x, t = _data(rng, 256)
        g, loss = net.grad(x, t)
        lref, gref = mo.loss_and_grad(p, DIMS, x.astype(np.float64), t.astype(np.float64))
        assert abs(loss - lref) <= 1e-3 * abs(lref)
        o = 0
        for l in range(len(DIMS) - 1):
            for n in (DIMS[l] * DIMS[l + 1], DIMS[l + 1]):
                a, r = g[o:o + n], gref[o:o + n]
                rel = np.linalg.norm(a - r) / max(np.linalg.norm(r), 1e-30)
                assert rel < 1e-2, (l, n, rel)
                o += n
        # parameters round-trip through the padded device copies
        q = p + np.float32(0.01)
        net.set_params(q)
        assert np.array_equal(net.get_params(), q)
    finally:
        net.close()


def test_inference_matches_oracle(built):
    rng = np.random.default_rng(2)
    net = built.Mlp(DIMS, seed=6)
    try:
        x, _ = _data(rng, 1000)
        y = net.forward(x)
        ref, _ = mo.forward(net.get_params(), DIMS, x.astype(np.float64))
        rel = np.linalg.norm(y - ref) / np.linalg.norm(ref)
        assert y.shape == (1000, DIMS[-1]) and rel < 1e-2, rel
    finally:
        net.close()


def test_training_reduces_loss(built):
    rng = np.random.default_rng(3)
    x, t = _data(rng, 8192)
    net = built.Mlp(DIMS, seed=7)
    try:
        losses, ms = net.train(x, t, epochs=40, lr=1e-3, seed=11)
        assert np.all(np.isfinite(losses)) and ms > 0
        assert losses[-1] < 0.2 * losses[0], losses[[0, 9, 19, 39]]
        y = net.forward(x[:1024])
        acc = np.mean((y[:, -1] > 0) == (t[:1024, -1] > 0.5))
        assert acc > 0.85, acc
    finally:
        net.close()


def test_large_inference_matches_oracle(built):
    # 40,000 rows = 313 row tiles: the persistent kernel (W resident, two TMEM
    # accumulators alternating, ragged last tile)
    rng = np.random.default_rng(4)
    net = built.Mlp(DIMS, seed=8)
    try:
        x, _ = _data(rng, 40000)
        y = net.forward(x)
        ref, _ = mo.forward(net.get_params(), DIMS, x.astype(np.float64))
        rel = np.linalg.norm(y - ref) / np.linalg.norm(ref)
        assert rel < 1e-2, rel
        # rows across the tile boundaries agree with a small (non-persistent) call
        for lo in (0, 127, 38656, 39936):
            ys = net.forward(x[lo:lo + 64])
            np.testing.assert_array_equal(ys, y[lo:lo + 64])
    finally:
        net.close()
