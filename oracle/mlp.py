"""CPU oracle of the surrogate network (test infrastructure: only tests and
bench.py's baseline legs use it).

The surrogate (bd_aging_b200/csrc/surrogate.cu) is an MLP n_in -> width x
depth (GELU, exact erf form) -> n_out with loss
    L = 1 / (B n_out) sum_b sum_n w_n (y_bn - t_bn)^2.
This module restates its forward and backward pass in FP64 numpy.  With
`bf16=True` it rounds where the GPU stores BF16 (inputs, weights,
activations, the loss gradient and every dZ), so GPU gradients can be
compared closely; with `bf16=False` it is the exact FP64 network, checked
against central finite differences."""
from __future__ import annotations

import math

import numpy as np


def to_bf16(x: np.ndarray) -> np.ndarray:
    """Round FP32/FP64 values to BF16 (nearest, ties to even), returned as float64."""
    f = np.ascontiguousarray(np.asarray(x, np.float64).astype(np.float32))
    u = f.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def bf16_bits(x: np.ndarray) -> np.ndarray:
    f = np.ascontiguousarray(np.asarray(x, np.float64).astype(np.float32))
    u = f.view(np.uint32).astype(np.uint64)
    return (((u + 0x7FFF + ((u >> 16) & 1)) >> 16) & 0xFFFF).astype(np.uint16)


_erf = np.vectorize(math.erf)


def gelu(z):
    return 0.5 * z * (1.0 + _erf(z / math.sqrt(2.0)))


def gelu_grad(z):
    return 0.5 * (1.0 + _erf(z / math.sqrt(2.0))) + z * np.exp(-0.5 * z * z) / math.sqrt(2.0 * math.pi)


def unflatten(params: np.ndarray, sizes):
    """sizes: [(N_l, K_l)] -> [(W_l [N][K], b_l [N])] from the flat layout of
    bd_surrogate_get_params (per layer W row-major, then b)."""
    out, off = [], 0
    for n, k in sizes:
        w = params[off:off + n * k].reshape(n, k)
        off += n * k
        b = params[off:off + n]
        off += n
        out.append((np.asarray(w, np.float64), np.asarray(b, np.float64)))
    return out


def flatten(layers) -> np.ndarray:
    return np.concatenate([np.concatenate([w.ravel(), b.ravel()]) for w, b in layers])


def sizes_of(n_in, n_out, width, depth):
    return [(width, n_in)] + [(width, width)] * (depth - 1) + [(n_out, width)]


def loss_and_grad(layers, x, t, w_out=None, bf16=False):
    """Mean weighted squared error and its gradient (same layout as layers)."""
    rnd = to_bf16 if bf16 else (lambda a: np.asarray(a, np.float64))
    B = x.shape[0]
    n_out = layers[-1][0].shape[0]
    w_out = np.ones(n_out) if w_out is None else np.asarray(w_out, np.float64)
    Wq = [rnd(w) for w, _ in layers]
    hs = [rnd(x)]
    zs = []
    for l, (w, b) in enumerate(layers):
        z = hs[-1] @ Wq[l].T + b
        zs.append(z)
        if l < len(layers) - 1:
            hs.append(rnd(gelu(z)))
    y = zs[-1]
    e = y - t
    loss = float((w_out * e * e).sum() / (B * n_out))
    dz = rnd(2.0 * w_out * e / (B * n_out))
    grads = [None] * len(layers)
    for l in range(len(layers) - 1, -1, -1):
        grads[l] = (dz.T @ hs[l], dz.sum(0))
        if l > 0:
            dh = dz @ Wq[l]
            dz = rnd(dh * gelu_grad(zs[l - 1]))
    return loss, grads, y


def predict(layers, x, bf16=False):
    rnd = to_bf16 if bf16 else (lambda a: np.asarray(a, np.float64))
    h = rnd(x)
    for l, (w, b) in enumerate(layers):
        z = h @ rnd(w).T + b
        h = rnd(gelu(z)) if l < len(layers) - 1 else z
    return h


def finite_difference(layers, x, t, idx, eps=1e-6):
    """Central differences of the FP64 loss for flat parameter indices idx."""
    flat = flatten(layers)
    sizes = [w.shape for w, _ in layers]
    out = []
    for i in idx:
        p = flat.copy()
        p[i] += eps
        lp, _, _ = loss_and_grad(unflatten(p, sizes), x, t)
        p[i] -= 2 * eps
        lm, _, _ = loss_and_grad(unflatten(p, sizes), x, t)
        out.append((lp - lm) / (2 * eps))
    return np.array(out)
