"""CPU oracle of the surrogate MLP's forward and backward passes (test
infrastructure only: tests/ import it to check the tensor-core kernels; the
product never does).

The surrogate has no counterpart in the reference, so this oracle is pinned
two ways instead: with rounding switched off its gradients agree with central
finite differences of its own loss (tests/test_mlp_oracle.py), and with
rounding on it applies BF16 round-to-nearest-even at exactly the points the
device kernels do (inputs, weights, hidden activations, output-layer and
hidden gradients), accumulating in float64 where the device accumulates in
FP32.

Layout of a parameter vector: per layer W [out x in] row-major, then b [out].
Loss of a batch of R rows with outputs y and targets t (the last column is
the hyperactivity label, the others log(1 + rate)):
    (1 / (R * nr)) * sum (y_r - t_r)^2  +  (1 / R) * sum BCE(y_logit, t_logit).
"""
from __future__ import annotations

from typing import List, Sequence, Tuple

import numpy as np


def bf16_bits(x: np.ndarray) -> np.ndarray:
    """float32 -> BF16 bit patterns, round to nearest even (finite inputs)."""
    u = np.ascontiguousarray(x, np.float32).view(np.uint32).astype(np.uint64)
    r = ((u >> 16) & 1) + 0x7FFF
    return ((u + r) >> 16).astype(np.uint16)


def bf16(x: np.ndarray) -> np.ndarray:
    """Values rounded to BF16 (as float64)."""
    b = bf16_bits(np.asarray(x, np.float32)).astype(np.uint32) << 16
    return b.view(np.float32).astype(np.float64)


def unpack(p: np.ndarray, dims: Sequence[int]) -> List[Tuple[np.ndarray, np.ndarray]]:
    out, o = [], 0
    for l in range(len(dims) - 1):
        n_in, n_out = dims[l], dims[l + 1]
        W = p[o:o + n_in * n_out].reshape(n_out, n_in).astype(np.float64)
        o += n_in * n_out
        b = p[o:o + n_out].astype(np.float64)
        o += n_out
        out.append((W, b))
    return out


def pack(layers) -> np.ndarray:
    return np.concatenate([np.concatenate([W.ravel(), b]) for W, b in layers]).astype(np.float64)


def forward(p, dims, X, rounding: bool = True):
    rd = bf16 if rounding else (lambda a: np.asarray(a, np.float64))
    layers = unpack(np.asarray(p), dims)
    h = rd(X)
    acts = [h]
    for l, (W, b) in enumerate(layers):
        z = h @ rd(W).T + b
        if l + 1 < len(layers):
            h = rd(np.maximum(z, 0.0))
            acts.append(h)
        else:
            return z, acts
    raise AssertionError


def loss_and_grad(p, dims, X, T, rounding: bool = True):
    rd = bf16 if rounding else (lambda a: np.asarray(a, np.float64))
    layers = unpack(np.asarray(p), dims)
    z, acts = forward(p, dims, X, rounding)
    R, nr = X.shape[0], dims[-1] - 1
    e = z[:, :nr] - T[:, :nr]
    y, t = z[:, nr], T[:, nr]
    loss = float((e * e).sum() / (R * nr) + (np.maximum(y, 0) - y * t + np.log1p(np.exp(-np.abs(y)))).sum() / R)
    dz = np.zeros_like(z)
    dz[:, :nr] = 2.0 * e / (R * nr)
    dz[:, nr] = (1.0 / (1.0 + np.exp(-y)) - t) / R
    dz = rd(dz)
    grads = [None] * len(layers)
    for l in range(len(layers) - 1, -1, -1):
        W, _ = layers[l]
        gW = dz.T @ acts[l]
        gb = dz.sum(0)
        grads[l] = (gW, gb)
        if l > 0:
            dz = rd((dz @ rd(W)) * (acts[l] > 0))
    return loss, pack(grads)
