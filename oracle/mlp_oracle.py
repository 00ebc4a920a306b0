"""FP64 CPU restatement of the warm-start network (TEST INFRASTRUCTURE ONLY).

The checker for the tensor-core MLP of cuopo_b200/csrc/mlp.cu: the same
network (n_in -> width GELU x depth -> n_out, mean squared error over all
outputs, Adam with beta1 0.9, beta2 0.999, eps 1e-8) in numpy float64.  The
reference has no network (it starts every run from noise,
src/headers/functions.cuh:58-71), so this oracle is pinned by a finite-
difference check of its own gradients (tests/test_mlp_oracle.py), not by
reference vectors.

With emulate_bf16=True the values that the GPU stores in BF16 are rounded
to BF16 at the same points: the input, the weights, the derivative
GELU'(z) of every hidden pre-activation (stored by the forward pass for the
backward one), the activations h, the output gradient and every
back-propagated gradient (the bias gradients sum the rounded values).  Sums
are exact (float64) either way, so the remaining difference from the GPU is
its FP32 accumulation order and its FP32 GELU (whose erf is a published
approximation with absolute error <= 1.5e-7, far below the BF16 rounding).

Parameter layout (flat): per layer l = 0..depth, W_l [N_l][K_l] row-major
then b_l [N_l]; N_l = width except the last (n_out), K_0 = n_in, else width.
"""
from __future__ import annotations

import numpy as np
from scipy.special import erf

SQRT1_2 = 0.70710678118654752440
INV_SQRT_2PI = 0.39894228040143267794


def bf16(a) -> np.ndarray:
    """Round to the nearest BF16 (ties to even), returned as float64."""
    f = np.ascontiguousarray(a, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def gelu(x):
    return 0.5 * x * (1.0 + erf(x * SQRT1_2))


def gelu_grad(x):
    return 0.5 * (1.0 + erf(x * SQRT1_2)) + x * INV_SQRT_2PI * np.exp(-0.5 * x * x)


def layer_dims(n_in: int, width: int, depth: int, n_out: int):
    """(N_l, K_l) for l = 0..depth."""
    return [(width if l < depth else n_out, n_in if l == 0 else width) for l in range(depth + 1)]


def param_count(dims) -> int:
    return sum(n * k + n for n, k in dims)


def unpack(params: np.ndarray, dims):
    out, o = [], 0
    for n, k in dims:
        W = params[o:o + n * k].reshape(n, k)
        o += n * k
        b = params[o:o + n]
        o += n
        out.append((W, b))
    return out


def pack(layers) -> np.ndarray:
    return np.concatenate([np.concatenate([W.ravel(), b.ravel()]) for W, b in layers])


def forward(params, x, dims, emulate_bf16: bool = True):
    """Returns (y, cache) for input x [B][n_in]."""
    r = bf16 if emulate_bf16 else (lambda a: np.asarray(a, np.float64))
    layers = unpack(np.asarray(params, np.float64), dims)
    a = r(x)
    cache = {"a": [a], "gp": []}
    for l, (W, b) in enumerate(layers):
        z = a @ r(W).T + b
        if l == len(layers) - 1:
            return z, cache
        cache["gp"].append(r(gelu_grad(z)))
        a = r(gelu(z))
        cache["a"].append(a)
    raise AssertionError("unreachable")


def loss_and_grads(params, x, t, dims, emulate_bf16: bool = True):
    """Mean squared error over B x n_out and its gradient (flat layout)."""
    r = bf16 if emulate_bf16 else (lambda a: np.asarray(a, np.float64))
    params = np.asarray(params, np.float64)
    layers = unpack(params, dims)
    y, cache = forward(params, x, dims, emulate_bf16)
    B, n_out = y.shape
    d = y - t
    loss = float(np.mean(d * d))
    g = r(d * (2.0 / (B * n_out)))
    grads = [None] * len(layers)
    for l in range(len(layers) - 1, -1, -1):
        W, _ = layers[l]
        a = cache["a"][l]
        gW = g.T @ a
        gb = g.sum(axis=0)
        grads[l] = (gW, gb)
        if l == 0:
            break
        g = r((g @ r(W)) * cache["gp"][l - 1])
    return loss, pack(grads)


def adam_step(params, grads, m, v, step: int, lr: float, beta1=0.9, beta2=0.999, eps=1e-8):
    """One Adam update in place (step counts from 1)."""
    m *= beta1
    m += (1 - beta1) * grads
    v *= beta2
    v += (1 - beta2) * grads * grads
    mh = m / (1 - beta1 ** step)
    vh = v / (1 - beta2 ** step)
    params -= lr * mh / (np.sqrt(vh) + eps)
    return params
