"""Test infrastructure only: CPU FP64 restatement of the spectrum-surrogate MLP.

The checker for the GPU ensemble in ``gdiamond_b200/csrc/mlp.cu`` (no reference counterpart:
gDiamond has no learned component).  Plain numpy in float64:

* ``forward`` / ``loss_and_grad``: x -> [Linear -> GELU]* -> Linear, mean-squared-error loss
  and its gradient by backpropagation.
* ``bf16=True`` applies the GPU's roundings at the same places -- inputs, weights, hidden
  activations and the back-propagated pre-activation gradients rounded to BF16 (nearest-even)
  before they enter a product -- and computes everything else exactly, so the GPU's FP32
  accumulation is the only remaining difference.
* ``adam``: one Adam step (bias-corrected, b1 0.9, b2 0.999, eps 1e-8).

Layers are lists of (W [out][in], b [out]) arrays.  Pinned by central finite differences of
the exact (bf16=False) loss.  Only tests/ use this module.
"""
from __future__ import annotations

import numpy as np
from scipy.special import erf

SQRT1_2 = 0.7071067811865476
INV_SQRT_2PI = 0.3989422804014327


def round_bf16(x):
    """float32 round-to-nearest-even to BF16, returned as float64."""
    b = np.asarray(x, np.float32).view(np.uint32).astype(np.uint64)
    r = ((b + 0x7FFF + ((b >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    return r.view(np.float32).astype(np.float64)


def gelu(z):
    return 0.5 * z * (1.0 + erf(z * SQRT1_2))


def gelu_grad(z):
    return 0.5 * (1.0 + erf(z * SQRT1_2)) + z * INV_SQRT_2PI * np.exp(-0.5 * z * z)


def _q(x, bf16):
    return round_bf16(x) if bf16 else np.asarray(x, np.float64)


def forward(layers, x, bf16=False):
    """Returns (y, cache): the output and what backprop needs."""
    a = _q(x, bf16)
    acts, zs = [a], []
    for n, (W, b) in enumerate(layers):
        z = a @ _q(W, bf16).T + np.asarray(b, np.float64)
        zs.append(z)
        if n + 1 < len(layers):
            a = gelu(z)
            if bf16:
                a = round_bf16(a.astype(np.float32))
            acts.append(a)
    return zs[-1], (acts, zs)


def loss_and_grad(layers, x, y, bf16=False):
    """Mean squared error over all outputs and its gradient [(dW, db)] per layer."""
    out, (acts, zs) = forward(layers, x, bf16)
    t = np.asarray(y, np.float64)
    M, N = out.shape
    d = out - t
    loss = float(np.mean(d * d))
    g = 2.0 * d / (M * N)
    grads = [None] * len(layers)
    for n in range(len(layers) - 1, -1, -1):
        W = layers[n][0]
        gq = round_bf16(g.astype(np.float32)) if bf16 else g
        grads[n] = (gq.T @ acts[n], g.sum(axis=0))
        if n > 0:
            g = (gq @ _q(W, bf16)) * gelu_grad(zs[n - 1])
    return loss, grads


def adam(params, grads, m, v, t, lr, b1=0.9, b2=0.999, eps=1e-8):
    """One Adam step on flat arrays (t = the step number, from 1); returns new (p, m, v)."""
    m = b1 * m + (1 - b1) * grads
    v = b2 * v + (1 - b2) * grads * grads
    p = params - lr * (m / (1 - b1 ** t)) / (np.sqrt(v / (1 - b2 ** t)) + eps)
    return p, m, v
