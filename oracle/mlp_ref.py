"""FP64 restatement of the coordinate MLP (TEST INFRASTRUCTURE ONLY): the
checker of the CUDA forward / backward kernels (include/rt_b200_mlp.h).

Same architecture and parameter layout: IN=8 -> 128 -> 128 -> 128 -> 1, GELU
(tanh form) after each hidden layer, mean squared error.  `bf16_like_gpu`
rounds the operands the GPU keeps in BF16 (the 128x128 weights and the
hidden activations / gradients entering the tensor-core GEMMs), so the
comparison isolates accumulation order from storage precision.
"""
from __future__ import annotations

import numpy as np

IN, H = 8, 128
SIZES = [("W0", (H, IN)), ("b0", (H,)), ("W1", (H, H)), ("b1", (H,)), ("W2", (H, H)), ("b2", (H,)),
         ("W3", (H,)), ("b3", (1,))]
NPARAM = sum(int(np.prod(s)) for _, s in SIZES)
C = 0.7978845608028654  # sqrt(2 / pi)


def unpack(p):
    out, at = {}, 0
    for name, shape in SIZES:
        k = int(np.prod(shape))
        out[name] = np.asarray(p[at:at + k], dtype=np.float64).reshape(shape)
        at += k
    return out


def bf16(x):
    """Round to bfloat16 (nearest even) and back, as __float2bfloat16 does."""
    a = np.asarray(x, dtype=np.float32).copy()
    u = a.view(np.uint32)
    u += 0x7FFF + ((u >> 16) & 1)
    u &= 0xFFFF0000
    return a.astype(np.float64)


def gelu(z):
    return 0.5 * z * (1.0 + np.tanh(C * (z + 0.044715 * z ** 3)))


def gelu_grad(z):
    t = np.tanh(C * (z + 0.044715 * z ** 3))
    return 0.5 * (1.0 + t) + 0.5 * z * (1.0 - t * t) * C * (1.0 + 3 * 0.044715 * z * z)


def loss_grad(params, x, target, bf16_like_gpu=True):
    P = unpack(params)
    r = bf16 if bf16_like_gpu else (lambda v: np.asarray(v, dtype=np.float64))
    x = np.asarray(x, dtype=np.float64)
    t = np.asarray(target, dtype=np.float64)
    n = x.shape[0]
    W1, W2 = r(P["W1"]), r(P["W2"])
    z0 = x @ P["W0"].T + P["b0"]
    h1 = r(gelu(z0))
    z1 = h1 @ W1.T + P["b1"]
    h2 = r(gelu(z1))
    z2 = h2 @ W2.T + P["b2"]
    h3 = r(gelu(z2))
    y = h3 @ P["W3"] + P["b3"][0]
    e = y - t
    loss = float(np.mean(e * e))
    dy = 2.0 * e / n
    g = {"W3": h3.T @ dy, "b3": np.array([dy.sum()])}
    dz2 = np.outer(dy, P["W3"]) * gelu_grad(z2)
    g["W2"] = r(dz2).T @ h2
    g["b2"] = dz2.sum(0)
    dz1 = (r(dz2) @ W2) * gelu_grad(z1)
    g["W1"] = r(dz1).T @ h1
    g["b1"] = dz1.sum(0)
    dz0 = (r(dz1) @ W1) * gelu_grad(z0)
    g["W0"] = dz0.T @ x
    g["b0"] = dz0.sum(0)
    flat = np.concatenate([g[name].reshape(-1) for name, _ in SIZES])
    return loss, flat, y
