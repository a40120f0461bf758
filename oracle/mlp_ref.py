"""TEST INFRASTRUCTURE ONLY: CPU restatement of the library's learned
self-energy network (edus_2.0_b200/csrc/surrogate.cu), the checker of its
forward pass and gradients.  No reference counterpart: the network is new.

The GPU multiplies BF16 operands (weights, the input, the hidden activations
and the back-propagated errors, each rounded to nearest even) with FP32
accumulation; this restatement rounds the same operands to BF16 and
multiplies in FP64, so the two differ only by the accumulation order and
precision.  Parameters are flattened as W0 b0 W1 b1 W2 b2 W3 b3, W_l
row-major [in][out]; activations GELU (erf form) after the three hidden
layers; loss mean((y - t)^2).
"""
import math

import numpy as np


def bf16(x):
    """Round to the nearest BF16 value (ties to even), returned as float64."""
    f = np.ascontiguousarray(x, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    return r.view(np.float32).astype(np.float64)


_erf = np.vectorize(math.erf)


def gelu(z):
    return 0.5 * z * (1.0 + _erf(z / math.sqrt(2.0)))


def gelu_grad(z):
    cdf = 0.5 * (1.0 + _erf(z / math.sqrt(2.0)))
    return cdf + z * np.exp(-0.5 * z * z) / math.sqrt(2.0 * math.pi)


def unflatten(p, dims):
    out, off = [], 0
    for i in range(len(dims) - 1):
        n = dims[i] * dims[i + 1]
        W = p[off:off + n].reshape(dims[i], dims[i + 1]).astype(np.float64)
        off += n
        b = p[off:off + dims[i + 1]].astype(np.float64)
        off += dims[i + 1]
        out.append((W, b))
    return out


def _ident(x):
    return np.asarray(x, dtype=np.float64)


def forward(p, dims, x, round_ops=True):
    """(output, pre-activations, operand activations).  round_ops=False keeps
    every operand in FP64 (for finite-difference checks of this file)."""
    q = bf16 if round_ops else _ident
    layers = unflatten(p, dims)
    a = q(x)
    zs, acts = [], [a]
    for i, (W, b) in enumerate(layers):
        z = acts[-1] @ q(W) + b
        if round_ops:
            z = z.astype(np.float32).astype(np.float64)
        zs.append(z)
        if i < len(layers) - 1:
            acts.append(q(gelu(z)))
    return zs[-1], zs, acts


def gradients(p, dims, x, t, round_ops=True):
    """(flattened gradient of mean((y - t)^2), loss)."""
    q = bf16 if round_ops else _ident
    layers = unflatten(p, dims)
    y, zs, acts = forward(p, dims, x, round_ops)
    n = y.size
    loss = float(np.sum((y - t) ** 2) / n)
    dz = 2.0 * (y - t) / n
    grads = [None] * len(layers)
    for i in range(len(layers) - 1, -1, -1):
        W, _ = layers[i]
        dzb = q(dz)
        gW = acts[i].T @ dzb
        gb = dz.sum(axis=0)
        grads[i] = (gW, gb)
        if i == 0:
            break
        da = dzb @ q(W).T
        dz = da * gelu_grad(zs[i - 1])
    flat = []
    for gW, gb in grads:
        flat.append(gW.ravel())
        flat.append(gb)
    return np.concatenate(flat), loss
