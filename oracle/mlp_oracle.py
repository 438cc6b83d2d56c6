"""NumPy restatement of the surrogate MLP's forward and backward pass.
TEST INFRASTRUCTURE ONLY: the checker for the tcgen05 training kernels.

It mirrors the GPU step's numerics point by point: weights, layer inputs and
back-propagated gradients are rounded to bf16 (round to nearest even) where
the GPU feeds them to the tensor cores, products are accumulated in FP32,
pre-activations, the loss and the bias gradients stay FP32.  Network:
nin -> H -> H -> H -> nout, exact GELU, weighted mean softmax cross-entropy.
Parameter vector layout: for each layer, W [out x in] row-major, then b [out].
"""
from __future__ import annotations

import numpy as np
from scipy.special import erf


def bf16(a: np.ndarray) -> np.ndarray:
    """Round float32 values to bfloat16 (nearest even), returned as float32."""
    a = np.ascontiguousarray(a, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    bias = ((u >> 16) & 1) + 0x7FFF
    r = ((u + bias) & 0xFFFF0000).astype(np.uint32)
    return r.view(np.float32)


def gelu(z):
    return (0.5 * z * (1.0 + erf(z * 0.70710678118654752))).astype(np.float32)


def dgelu(z):
    return (0.5 * (1.0 + erf(z * 0.70710678118654752)) + z * 0.39894228040143268 * np.exp(-0.5 * z * z)).astype(np.float32)


def unpack(params: np.ndarray, nin: int, H: int, nout: int):
    dims = [(H, nin), (H, H), (H, H), (nout, H)]
    out, off = [], 0
    for o, i in dims:
        W = params[off:off + o * i].reshape(o, i)
        off += o * i
        b = params[off:off + o]
        off += o
        out.append((W, b))
    return out


def forward_backward(params, x, labels, weights, nin, H, nout):
    """Returns (loss, probs, grads) with grads in the parameter layout."""
    layers = unpack(np.asarray(params, dtype=np.float32), nin, H, nout)
    x = np.asarray(x, dtype=np.float32)
    B = x.shape[0]
    w = np.ones(B, np.float32) if weights is None else np.asarray(weights, np.float32)
    norm = np.float32(w.sum())
    acts = [bf16(x)]
    Zs = []
    h = acts[0]
    for l in range(3):
        W, b = layers[l]
        z = (h @ bf16(W).T).astype(np.float32) + b
        Zs.append(z)
        h = bf16(gelu(z))
        acts.append(h)
    W4, b4 = layers[3]
    logits = (h @ bf16(W4).T).astype(np.float32) + b4
    m = logits.max(axis=1, keepdims=True)
    e = np.exp(logits - m)
    s = e.sum(axis=1, keepdims=True)
    p = e / s
    onehot = np.zeros_like(p)
    onehot[np.arange(B), labels] = 1.0
    loss = float((w * (np.log(s[:, 0]) + m[:, 0] - logits[np.arange(B), labels])).sum() / norm)
    dz = (w[:, None] * (p - onehot) / norm).astype(np.float32)
    grads = []
    for l in range(3, -1, -1):
        W, b = layers[l]
        dzb = bf16(dz)
        gW = (dzb.T @ acts[l]).astype(np.float32)
        gb = dz.sum(axis=0).astype(np.float32)
        grads.append((gW, gb))
        if l > 0:
            dh = (dzb @ bf16(W)).astype(np.float32)
            dz = (dh * dgelu(Zs[l - 1])).astype(np.float32)
    grads = grads[::-1]
    flat = np.concatenate([np.concatenate([g.ravel(), gb]) for g, gb in grads])
    return loss, p, flat


def init_params(nin, H, nout, seed=0):
    rng = np.random.default_rng(seed)
    dims = [(H, nin), (H, H), (H, H), (nout, H)]
    parts = []
    for o, i in dims:
        a = 1.0 / np.sqrt(i)
        parts.append(rng.uniform(-a, a, o * i))
        parts.append(rng.uniform(-a, a, o))
    return np.concatenate(parts).astype(np.float32)
