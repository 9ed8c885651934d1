"""CPU ORACLE of the learned surrogate's network -- test infrastructure only.

A numpy restatement of the multilayer perceptron of the library's surrogate
(n_in -> width x depth, GELU -> n_out, weighted mean-square error) with its forward pass,
the backward pass to every parameter and to the inputs, and Adam.  ``bf16=True`` rounds the
operands of every matrix product to bfloat16 exactly where the GPU does (the packed inputs,
the activations, the weights and the backward signals) and accumulates in FP64, so the GPU's
FP32-accumulated tensor-core products can be checked to FP32 rounding; ``bf16=False`` is the
plain FP64 network.

Only ``tests/`` imports this module.
"""
from __future__ import annotations

import numpy as np
from scipy.special import erf


def bf16(a):
    """Round to bfloat16 (round to nearest, ties to even), returned as float64."""
    f = np.ascontiguousarray(a, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def gelu(x):
    return 0.5 * x * (1.0 + erf(x / np.sqrt(2.0)))


def gelu_d(x):
    return 0.5 * (1.0 + erf(x / np.sqrt(2.0))) + x * np.exp(-0.5 * x * x) / np.sqrt(2.0 * np.pi)


def unflatten(params, widths):
    """Split the flat parameter vector (W_l row-major then b_l, layer by layer)."""
    out, o = [], 0
    for k, n in zip(widths[:-1], widths[1:]):
        W = np.asarray(params[o:o + n * k], dtype=np.float64).reshape(n, k)
        o += n * k
        b = np.asarray(params[o:o + n], dtype=np.float64)
        o += n
        out.append((W, b))
    return out


def forward(params, widths, X, bf16_ops=True):
    rnd = bf16 if bf16_ops else (lambda a: np.asarray(a, dtype=np.float64))
    layers = unflatten(params, widths)
    H = rnd(X)
    Zs, Hs = [], [H]
    for i, (W, b) in enumerate(layers):
        Z = H @ rnd(W).T + b
        Zs.append(Z)
        if i + 1 < len(layers):
            H = rnd(gelu(Z))
            Hs.append(H)
    return Zs[-1], Zs, Hs


def loss_grad(params, widths, X, T, w_out=None, bf16_ops=True):
    """Loss sum_j w_j (y - t)^2 / (B n_out), gradients w.r.t. the flat parameters and X."""
    rnd = bf16 if bf16_ops else (lambda a: np.asarray(a, dtype=np.float64))
    layers = unflatten(params, widths)
    Y, Zs, Hs = forward(params, widths, X, bf16_ops)
    B, n = Y.shape
    w = np.ones(n) if w_out is None else np.asarray(w_out, dtype=np.float64)
    d = Y - T
    loss = float(np.sum(w * d * d) / (B * n))
    dZ = 2.0 * w * d / (B * n)
    grads = [None] * len(layers)
    dX = None
    for i in range(len(layers) - 1, -1, -1):
        W, _ = layers[i]
        dZr = rnd(dZ)
        gW = dZr.T @ Hs[i]
        gb = dZ.sum(axis=0)
        grads[i] = (gW, gb)
        dH = dZr @ rnd(W)
        if i == 0:
            dX = dH
        else:
            dZ = dH * gelu_d(Zs[i - 1])
    flat = np.concatenate([np.concatenate([gW.ravel(), gb]) for gW, gb in grads])
    return loss, flat, dX
