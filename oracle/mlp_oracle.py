"""CPU oracle (numpy, FP64) of the surrogate MLP.

TEST INFRASTRUCTURE ONLY: the checker of the CUDA forward/backward/Adam
kernels of ``csrc/surrogate.cu``; the product never imports it.  The
surrogate has no counterpart in the reference, so this module restates the
network the library defines (its parameter layout and arithmetic) in FP64:

* linear layers y = x W^T + b with W rounded to BF16 (round to nearest even,
  as ``__float2bfloat16_rn``) and b in FP32; SiLU z * sigmoid(z) after every
  hidden layer;
* loss = mean over all n x n_out entries of (y - t)^2;
* Adam with bias correction on FP32 master weights.
"""
from __future__ import annotations

import numpy as np


def bf16_round(a):
    """Round FP32 values to the nearest BF16 value (ties to even), as FP32."""
    a = np.ascontiguousarray(np.asarray(a, dtype=np.float32))
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    return r.view(np.float32)


def layer_shapes(n_in, n_hidden, n_layers, n_out):
    return [(n_in if l == 0 else n_hidden, n_out if l == n_layers else n_hidden) for l in range(n_layers + 1)]


def unpack(params, shapes):
    """Split the parameter vector into [(W [out x in], b [out])]."""
    out = []
    o = 0
    for fi, fo in shapes:
        W = params[o:o + fi * fo].reshape(fo, fi)
        o += fi * fo
        b = params[o:o + fo]
        o += fo
        out.append((W, b))
    assert o == params.size
    return out


def _silu(z):
    return z / (1.0 + np.exp(-z))


def _dsilu(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def forward(params, shapes, X, keep=False):
    layers = unpack(np.asarray(params, np.float32), shapes)
    a = np.asarray(X, np.float64)
    cache = []
    for l, (W, b) in enumerate(layers):
        Wq = bf16_round(W).astype(np.float64)
        z = a @ Wq.T + b.astype(np.float64)
        cache.append((a, z, Wq))
        a = _silu(z) if l + 1 < len(layers) else z
    return (a, cache) if keep else a


def loss_grad(params, shapes, X, T):
    """MSE loss and its gradient with respect to the parameter vector."""
    Y, cache = forward(params, shapes, X, keep=True)
    T = np.asarray(T, np.float64)
    n = Y.size
    loss = float(np.sum((Y - T) ** 2) / n)
    dz = 2.0 * (Y - T) / n
    grads = []
    for l in range(len(cache) - 1, -1, -1):
        a, z, Wq = cache[l]
        if l + 1 < len(cache):
            dz = dz * _dsilu(z)
        gW = dz.T @ a
        gb = dz.sum(axis=0)
        grads.append((gW, gb))
        dz = dz @ Wq
    grads.reverse()
    return loss, np.concatenate([np.concatenate([gW.ravel(), gb]) for gW, gb in grads])


def adam_step(w, g, m, v, t, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8, wd=0.0):
    """One Adam step (t = 1, 2, ...); returns new (w, m, v)."""
    g = g + wd * w
    m = b1 * m + (1 - b1) * g
    v = b2 * v + (1 - b2) * g * g
    w = w - lr * (m / (1 - b1 ** t)) / (np.sqrt(v / (1 - b2 ** t)) + eps)
    return w, m, v
