"""CPU oracle of the learned face-flux network (test infrastructure only).

FP64 numpy forward and backward passes of the SmeLU MLP that the library trains on the
GPU (17 inputs, hidden layers of one width, 8 outputs; 17 -> 64 -> 64 -> 8 by default, any
other shape through the ``shp`` argument, e.g. ``shapes(128, 3)``), with the mean-squared-error loss and the Adam
update.  The GPU stores weights, activations and back-propagated errors in BF16 between
its tensor-core products; with ``bf16=True`` this oracle rounds the same quantities at
the same points (round-to-nearest-even of the FP32 value), so the two differ only by
accumulation order.  With ``bf16=False`` it is the exact FP64 network, checked against
finite differences by the tests.

The network has no counterpart in the reference (whose face solver,
src/modules/solvers/solver.f90:163-187, is always exact); HLLD (solver.f90:618-836) is
its label generator.  Parameter order: W1[17][64], b1[64], W2[64][64], b2, W3[64][8], b3
at the default shape; W1, b1, the hidden W[w][w], b pairs, then W[w][8], b in general (W[k][n] maps
input k to output n).
"""
from __future__ import annotations

import numpy as np

def shapes(width: int = 64, depth: int = 2) -> list[tuple[int, int]]:
    """(inputs, outputs) of each weight layer for `depth` hidden layers of `width` units."""
    return [(17, width)] + [(width, width)] * (depth - 1) + [(width, 8)]


SHAPES = shapes()


def unpack(p: np.ndarray, shp=None) -> list[tuple[np.ndarray, np.ndarray]]:
    out, off = [], 0
    for k, n in (shp or SHAPES):
        w = np.asarray(p[off:off + k * n], dtype=np.float64).reshape(k, n)
        off += k * n
        b = np.asarray(p[off:off + n], dtype=np.float64)
        off += n
        out.append((w, b))
    return out


def pack(layers: list[tuple[np.ndarray, np.ndarray]]) -> np.ndarray:
    return np.concatenate([np.concatenate([w.ravel(), b.ravel()]) for w, b in layers])


def bf16(a: np.ndarray) -> np.ndarray:
    """Round to BF16 (nearest even) through FP32, returned as float64."""
    f = np.asarray(a, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def smelu(z: np.ndarray) -> np.ndarray:
    """SmeLU with half-width 1 (Shamir et al. 2020), as the library uses it:
    0 for z <= -1, (z + 1)^2 / 4 for |z| < 1, z for z >= 1."""
    return np.where(z >= 1.0, z, np.where(z <= -1.0, 0.0, 0.25 * (z + 1.0) ** 2))


def smelu_d(z: np.ndarray) -> np.ndarray:
    return np.clip(0.5 * (z + 1.0), 0.0, 1.0)


def forward(p: np.ndarray, x: np.ndarray, bf16_rounding: bool = True, shp=None):
    """Network outputs and the cache needed by ``backward``."""
    r = bf16 if bf16_rounding else (lambda a: np.asarray(a, dtype=np.float64))
    layers = unpack(p, shp)
    h = r(x)
    cache = {"h": [h], "gd": [], "w": []}
    for l, (w, b) in enumerate(layers):
        wb = r(w)
        cache["w"].append(wb)
        z = h @ wb + b
        if l < len(layers) - 1:
            cache["gd"].append(smelu_d(z))
            h = r(smelu(z))
            cache["h"].append(h)
        else:
            y = z
    return y, cache


def loss_and_grad(p: np.ndarray, x: np.ndarray, t: np.ndarray, bf16_rounding: bool = True, shp=None):
    """Mean squared error over all outputs and its gradient in parameter order."""
    r = bf16 if bf16_rounding else (lambda a: np.asarray(a, dtype=np.float64))
    y, c = forward(p, x, bf16_rounding, shp)
    e = y - t
    loss = float(np.mean(e * e))
    d = 2.0 * e / e.size  # dL/dy
    nl = len(c["w"])
    grads = [None] * nl
    for l in range(nl - 1, -1, -1):
        db = d.sum(axis=0)
        dr = r(d)
        dw = c["h"][l].T @ dr
        grads[l] = (dw, db)
        if l > 0:
            d = (dr @ c["w"][l].T) * c["gd"][l - 1]
    return loss, pack(grads)


def adam_step(p, g, m, v, step, lr=1e-3, beta1=0.9, beta2=0.999, eps=1e-8):
    """One Adam update (step counts from 1); returns new (p, m, v)."""
    m = beta1 * m + (1 - beta1) * g
    v = beta2 * v + (1 - beta2) * g * g
    p = p - lr * (m / (1 - beta1 ** step)) / (np.sqrt(v / (1 - beta2 ** step)) + eps)
    return p, m, v
