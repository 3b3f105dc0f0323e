"""FP64 numpy restatement of the warm-start MLP (TEST INFRASTRUCTURE ONLY).

The checker of fastmbcui_b200's mbc_mlp_* kernels: the same layers
(tanh hidden, linear output), the same parameter layout (per layer W
row-major out x in, then b), the same loss 0.5 * mean((y - t)^2).  The
forward pass uses the weights rounded to BF16, as the kernels do.
"""
from __future__ import annotations

import numpy as np


def bf16_round(a: np.ndarray) -> np.ndarray:
    """Round FP32 values to BF16 (round to nearest even), returned as float64."""
    a = np.ascontiguousarray(a, np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    lsb = (u >> 16) & 1
    r = ((u + 0x7FFF + lsb) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(params: np.ndarray, dims):
    out, off = [], 0
    for l in range(len(dims) - 1):
        n, k = dims[l + 1], dims[l]
        W = params[off:off + n * k].reshape(n, k)
        off += n * k
        b = params[off:off + n]
        off += n
        out.append((W, b))
    assert off == params.size
    return out


def forward(params, dims, X):
    layers = unpack(np.asarray(params, np.float32), dims)
    acts = [np.asarray(X, np.float64)]
    for l, (W, b) in enumerate(layers):
        z = acts[-1] @ bf16_round(W).T + b.astype(np.float64)
        acts.append(z if l == len(layers) - 1 else np.tanh(z))
    return acts


def loss_and_grad(params, dims, X, T):
    """0.5 * mean((y - t)^2) and its gradient with respect to the parameters
    (taken through the BF16-rounded weights, as the kernels do)."""
    layers = unpack(np.asarray(params, np.float32), dims)
    acts = forward(params, dims, X)
    Y = acts[-1]
    T = np.asarray(T, np.float64)
    cnt = Y.size
    loss = 0.5 * np.sum((Y - T) ** 2) / cnt
    G = (Y - T) / cnt
    grads = []
    for l in range(len(layers) - 1, -1, -1):
        W, _ = layers[l]
        gW = G.T @ acts[l]
        gb = G.sum(axis=0)
        grads.append((gW, gb))
        if l > 0:
            G = (G @ bf16_round(W)) * (1.0 - acts[l] ** 2)
    grads.reverse()
    flat = np.concatenate([np.concatenate([gW.ravel(), gb]) for gW, gb in grads])
    return loss, flat
