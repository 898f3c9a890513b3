"""FP64 reference of the warm-start MLP (test infrastructure: the checker).

Mirrors the tensor-core kernels of the library: operands rounded to BF16 where
the kernels store BF16 (inputs, weights, hidden activations, backward
operands dO, dZ2, dZ1), FP64 products standing in for the FP32 tensor-core
accumulation, FP32-style bias and SiLU.  Parameter layout (FE_MODEL_PARAMS):
w1[64][16], w2[64][64], w3[2][64], b1[64], b2[64], b3[2].
"""
from __future__ import annotations

import numpy as np

W1, W2, W3 = 64 * 16, 64 * 64, 2 * 64
NW = W1 + W2 + W3
NP = NW + 64 + 64 + 2


def bf16(a) -> np.ndarray:
    """Round to the nearest BF16 (ties to even), returned as float64."""
    a = np.asarray(a, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    rounded = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    out = rounded.astype(np.uint32).view(np.float32).astype(np.float64)
    return np.where(np.isnan(a), np.nan, out)


def unpack(p):
    p = np.asarray(p, dtype=np.float64)
    w1 = p[:W1].reshape(64, 16)
    w2 = p[W1:W1 + W2].reshape(64, 64)
    w3 = p[W1 + W2:NW].reshape(2, 64)
    b1 = p[NW:NW + 64]
    b2 = p[NW + 64:NW + 128]
    b3 = p[NW + 128:NW + 130]
    return w1, w2, w3, b1, b2, b3


def silu(z):
    return z / (1.0 + np.exp(-z))


def silu_grad(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def pad16(x):
    x = np.asarray(x, dtype=np.float64)
    out = np.zeros((x.shape[0], 16))
    out[:, :x.shape[1]] = x
    return out


def forward(p, xs, quantize=True):
    """xs: standardised features [n][12].  Returns (out[n][2], cache)."""
    q = bf16 if quantize else (lambda a: np.asarray(a, dtype=np.float64))
    w1, w2, w3, b1, b2, b3 = unpack(p)
    X = q(pad16(xs))
    z1 = X @ q(w1).T + b1
    h1 = q(silu(z1))
    z2 = h1 @ q(w2).T + b2
    h2 = q(silu(z2))
    out = h2 @ q(w3).T + b3
    return out, (X, z1, h1, z2, h2)


def gradients(p, xs, ys, quantize=True):
    """Gradients of mean((out - ys)^2 summed over the 2 outputs) and the
    summed squared error, as the kernels compute them."""
    q = bf16 if quantize else (lambda a: np.asarray(a, dtype=np.float64))
    w1, w2, w3, b1, b2, b3 = unpack(p)
    n = xs.shape[0]
    out, (X, z1, h1, z2, h2) = forward(p, xs, quantize)
    ys = np.asarray(ys, dtype=np.float64)
    e = np.where(np.isnan(ys), 0.0, out - ys)   # NaN target: output not trained
    g = 2.0 * e / n
    gq = q(g)
    dh2 = gq @ q(w3)
    dz2 = dh2 * silu_grad(z2)
    dz2q = q(dz2)
    dh1 = dz2q @ q(w2)
    dz1 = dh1 * silu_grad(z1)
    dz1q = q(dz1)
    gw3 = gq.T @ h2
    gw2 = dz2q.T @ h1
    gw1 = dz1q.T @ X
    grads = np.concatenate([gw1.ravel(), gw2.ravel(), gw3.ravel(), dz1.sum(0), dz2.sum(0),
                            g.sum(0)])
    gw1_cols = grads[:W1].reshape(64, 16)
    gw1_cols[:, 12:] = 0.0
    return grads, float((e * e).sum())


def loss(p, xs, ys):
    out, _ = forward(p, xs, quantize=False)
    return float(((out - ys) ** 2).sum(1).mean())
