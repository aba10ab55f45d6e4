"""TEST INFRASTRUCTURE ONLY — FP64 numpy restatement of the equilibrium surrogate network
(3 -> 64 -> 64 -> 64 -> 4, GELU in its tanh form (Hendrycks & Gimpel 2016), mean-squared loss
over the 4 outputs) with the same flat parameter layout as the device code, used to check the
device forward / backward kernels:

    W1[3][64] b1[64] W2[64][64] b2[64] W3[64][64] b3[64] W4[64][4] b4[4]   (W in x out)

`forward_bf16` emulates the device inference: BF16 (round-to-nearest-even) weights and layer
inputs, FP32-like accumulation carried in FP64.
"""
from __future__ import annotations

import numpy as np

SIZES = [(3, 64), (64, 64), (64, 64), (64, 4)]
NPARAM = sum(k * n + n for k, n in SIZES)


def unpack(p: np.ndarray):
    p = np.asarray(p, dtype=np.float64)
    out, o = [], 0
    for k, n in SIZES:
        W = p[o:o + k * n].reshape(k, n)
        o += k * n
        b = p[o:o + n]
        o += n
        out.append((W, b))
    assert o == NPARAM
    return out


C = np.sqrt(2.0 / np.pi)
A = 0.044715


def gelu(z):
    return 0.5 * z * (1.0 + np.tanh(C * (z + A * z ** 3)))


def gelu_d(z):
    th = np.tanh(C * (z + A * z ** 3))
    return 0.5 * (1.0 + th) + 0.5 * z * (1.0 - th * th) * C * (1.0 + 3.0 * A * z * z)


def forward(p, X):
    layers = unpack(p)
    a = np.asarray(X, dtype=np.float64)
    zs, acts = [], [a]
    for i, (W, b) in enumerate(layers):
        z = a @ W + b
        zs.append(z)
        a = gelu(z) if i < len(layers) - 1 else z
        acts.append(a)
    return a, zs, acts


def loss_grad(p, X, T):
    """Mean squared error over all outputs and its gradient in the flat layout."""
    layers = unpack(p)
    Y, zs, acts = forward(p, X)
    cnt = Y.size
    d = Y - np.asarray(T, dtype=np.float64)
    loss = float((d * d).sum() / cnt)
    dz = 2.0 * d / cnt
    grads = [None] * len(layers)
    for i in range(len(layers) - 1, -1, -1):
        W, _ = layers[i]
        grads[i] = (acts[i].T @ dz, dz.sum(axis=0))
        if i > 0:
            dz = (dz @ W.T) * gelu_d(zs[i - 1])
    g = np.concatenate([np.concatenate([gw.ravel(), gb]) for gw, gb in grads])
    return loss, g


def bf16(x):
    """Round float32 values to bfloat16 (nearest even) and return them as float64."""
    a = np.ascontiguousarray(np.asarray(x, dtype=np.float32))
    u = a.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) >> 16
    return (u.astype(np.uint32) << 16).view(np.float32).astype(np.float64)


def forward_bf16(p, X):
    layers = unpack(p)
    a = np.asarray(X, dtype=np.float64)
    for i, (W, b) in enumerate(layers):
        z = bf16(a) @ bf16(W) + b.astype(np.float32).astype(np.float64)
        a = gelu(z) if i < len(layers) - 1 else z
    return a
