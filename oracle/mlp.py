"""CPU restatement of the warm-start MLP (test infrastructure only).

NumPy FP32 forward and backward of the network the tensor-core kernels run
(``co_cultivation_metabolic_atlas_b200/warmstart.py``), with the same BF16
rounding points: layer inputs (activations, upstream gradients) and weights
are rounded to BF16 before every product, products accumulate in FP32, and
pre-activations / gradients elsewhere stay FP32.  GELU is the erf form.
The reference's model is a torch MLP (``src/temporal_lp_model.py:58-142``)
trained with Adam on an MSE loss (``scripts/train_temporal_lp.py:23-88``).
"""

from __future__ import annotations

import math

import numpy as np


def bf16(x):
    """Round FP32 to the nearest BF16 (ties to even), returned as FP32."""
    a = np.ascontiguousarray(x, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    lsb = (u >> 16) & 1
    r = ((u + 0x7FFF + lsb) >> 16) << 16
    out = r.astype(np.uint32).view(np.float32)
    return np.where(np.isnan(a), a, out).astype(np.float32)


_erf = np.vectorize(math.erf, otypes=[np.float64])


def gelu(z):
    return (0.5 * z * (1.0 + _erf(z / math.sqrt(2.0)))).astype(np.float32)


def gelu_grad(z):
    z64 = z.astype(np.float64)
    cdf = 0.5 * (1.0 + _erf(z64 / math.sqrt(2.0)))
    pdf = np.exp(-0.5 * z64 * z64) / math.sqrt(2.0 * math.pi)
    return (cdf + z64 * pdf).astype(np.float32)


def forward(W, b, X, rounding=True):
    """W: list of (out, in) FP32 arrays (already the kernels' BF16 copies),
    b: biases, X: (B, in) FP32.  Returns output and the cache.  With
    ``rounding=False`` the same network runs in plain float64 (used to pin the
    backward pass against finite differences)."""
    rnd = bf16 if rounding else (lambda a: np.asarray(a, dtype=np.float64))
    h = rnd(X)
    dt = np.float32 if rounding else np.float64
    hs, zs = [h], []
    for l in range(len(W)):
        z = (h.astype(dt) @ rnd(W[l]).T.astype(dt)) + b[l]
        if l == len(W) - 1:
            return z.astype(dt), (hs, zs, rounding)
        zs.append(z.astype(dt))
        h = rnd(gelu(z) if rounding else _gelu64(z))
        hs.append(h)


def _gelu64(z):
    return 0.5 * z * (1.0 + _erf(z / math.sqrt(2.0)))


def backward(W, cache, dY):
    hs, zs, rounding = cache
    rnd = bf16 if rounding else (lambda a: np.asarray(a, dtype=np.float64))
    dt = np.float32 if rounding else np.float64
    gW = [None] * len(W)
    gb = [None] * len(W)
    dz = dY.astype(dt)
    for l in reversed(range(len(W))):
        dz16 = rnd(dz)
        gW[l] = (dz16.T @ hs[l]).astype(dt)
        gb[l] = dz.sum(axis=0).astype(dt)
        if l > 0:
            dh = (dz16 @ rnd(W[l])).astype(dt)
            gg = gelu_grad(zs[l - 1]) if rounding else gelu_grad(zs[l - 1]).astype(np.float64)
            dz = (dh * gg).astype(dt)
    return gW, gb
