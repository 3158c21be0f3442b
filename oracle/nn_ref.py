"""CPU oracle of the learned surrogate's operations (test infrastructure).

Plain numpy FP64 (or FP32) restatements of what pllcart3d_b200/csrc/nn.cu
computes, in the same channels-last layout ([n][d][h][w][c]) and weight
layout ([cout][tap][cin], tap = (dz*3 + dy)*3 + dx, offsets -1..1):
convolution forward, input and weight gradients, bias gradient, leaky ReLU,
2x average pooling, 2x nearest upsampling, concatenation, MSE and Adam.
Only tests import this module.
"""

from __future__ import annotations

import numpy as np


def _taps(k):
    if k == 1:
        return [(0, 0, 0)]
    return [(dz, dy, dx) for dz in range(3) for dy in range(3) for dx in range(3)]


def conv_fwd(x, w, b=None, k=3):
    """x [N,D,H,W,Ci], w [Co,k^3,Ci] -> [N,D,H,W,Co] (zero padding)."""
    N, D, H, W, Ci = x.shape
    Co = w.shape[0]
    p = (k - 1) // 2
    xp = np.pad(x, ((0, 0), (p, p), (p, p), (p, p), (0, 0)))
    y = np.zeros((N, D, H, W, Co), dtype=np.float64)
    for t, (dz, dy, dx) in enumerate(_taps(k)):
        y += xp[:, dz:dz + D, dy:dy + H, dx:dx + W, :] @ w[:, t, :].T
    if b is not None:
        y += b
    return y


def conv_bwd(x, w, gz, k=3):
    """Gradients of conv_fwd given dL/dz: (dx, dw, db)."""
    N, D, H, W, Ci = x.shape
    p = (k - 1) // 2
    xp = np.pad(x, ((0, 0), (p, p), (p, p), (p, p), (0, 0)))
    dxp = np.zeros_like(xp, dtype=np.float64)
    dw = np.zeros_like(w, dtype=np.float64)
    g2 = gz.reshape(-1, gz.shape[-1])
    for t, (dz, dy, dx) in enumerate(_taps(k)):
        xs = xp[:, dz:dz + D, dy:dy + H, dx:dx + W, :].reshape(-1, Ci)
        dw[:, t, :] = g2.T @ xs
        dxp[:, dz:dz + D, dy:dy + H, dx:dx + W, :] += gz @ w[:, t, :]
    dx_ = dxp[:, p:p + D, p:p + H, p:p + W, :]
    return dx_, dw, g2.sum(axis=0)


def leaky(z, slope):
    return np.where(z > 0, z, slope * z)


def leaky_bwd(z, g, slope):
    return np.where(z > 0, g, slope * g)


def pool(x):
    N, D, H, W, C = x.shape
    return x.reshape(N, D // 2, 2, H // 2, 2, W // 2, 2, C).mean(axis=(2, 4, 6))


def pool_bwd(g):
    return np.repeat(np.repeat(np.repeat(g, 2, axis=1), 2, axis=2), 2, axis=3) / 8.0


def up(x):
    return np.repeat(np.repeat(np.repeat(x, 2, axis=1), 2, axis=2), 2, axis=3)


def up_bwd(g):
    N, D, H, W, C = g.shape
    return g.reshape(N, D // 2, 2, H // 2, 2, W // 2, 2, C).sum(axis=(2, 4, 6))


def adam(w, g, m, v, lr, b1, b2, eps, t):
    m = b1 * m + (1 - b1) * g
    v = b2 * v + (1 - b2) * g * g
    w = w - lr * (m / (1 - b1 ** t)) / (np.sqrt(v / (1 - b2 ** t)) + eps)
    return w, m, v


# ---- the U-Net (same topology as pllcart3d_b200/surrogate.py) -------------

LAYERS = (("e1", 16, 32, 3, 1), ("e2", 32, 64, 3, 1), ("e3", 64, 128, 3, 1), ("e4", 128, 256, 3, 1),
          ("d3", 384, 128, 3, 1), ("d2", 192, 64, 3, 1), ("d1", 96, 32, 3, 1), ("out", 32, 16, 1, 0))


def unet_forward(params, x, slope, widths=None):
    """params: name -> (w, b); returns (out, cache)."""
    c = {}

    def conv(name, inp):
        w, b = params[name]
        k = 3 if w.shape[1] == 27 else 1
        z = conv_fwd(inp, w, b, k)
        act = dict((l[0], l[4]) for l in LAYERS)[name]
        y = leaky(z, slope) if act else z
        c[name] = (inp, z)
        return y

    e1 = conv("e1", x)
    e2 = conv("e2", pool(e1))
    e3 = conv("e3", pool(e2))
    e4 = conv("e4", pool(e3))
    d3 = conv("d3", np.concatenate([up(e4), e3], axis=-1))
    d2 = conv("d2", np.concatenate([up(d3), e2], axis=-1))
    d1 = conv("d1", np.concatenate([up(d2), e1], axis=-1))
    out = conv("out", d1)
    return out, c


def unet_backward(params, cache, gout, slope):
    grads = {}
    acts = dict((l[0], l[4]) for l in LAYERS)

    def back(name, gy):
        inp, z = cache[name]
        w, b = params[name]
        k = 3 if w.shape[1] == 27 else 1
        gz = leaky_bwd(z, gy, slope) if acts[name] else gy
        dx, dw, db = conv_bwd(inp, w, gz, k)
        grads[name] = (dw, db)
        return dx

    gd1 = back("out", gout)
    gc1 = back("d1", gd1)
    gu1, ge1 = gc1[..., :64], gc1[..., 64:]
    gc2 = back("d2", up_bwd(gu1))
    gu2, ge2 = gc2[..., :128], gc2[..., 128:]
    gc3 = back("d3", up_bwd(gu2))
    gu3, ge3 = gc3[..., :256], gc3[..., 256:]
    ge3 = ge3 + pool_bwd(back("e4", up_bwd(gu3)))
    ge2 = ge2 + pool_bwd(back("e3", ge3))
    ge1 = ge1 + pool_bwd(back("e2", ge2))
    back("e1", ge1)
    return grads
