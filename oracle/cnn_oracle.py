"""FP64 numpy restatement of the closure network (test infrastructure only; the checker of the
CUDA forward/backward/Adam kernels).  Same conventions as optimizec_b200/csrc/cnn.cuh:
activations [B][C][H][W], periodic 3x3 convolutions, parameters per layer = weights
[Co][Ci][3][3] then bias [Co], GELU(x) = x Phi(x) after every layer except the last, loss =
mean squared error."""
from __future__ import annotations

import numpy as np
from scipy.special import erf


def layer_shapes(layers: int, channels: int):
    return [(3 if l == 0 else channels, 1 if l == layers - 1 else channels) for l in range(layers)]


def unpack(params: np.ndarray, layers: int, channels: int):
    out, off = [], 0
    for ci, co in layer_shapes(layers, channels):
        w = params[off:off + co * ci * 9].reshape(co, ci, 3, 3)
        off += co * ci * 9
        b = params[off:off + co]
        off += co
        out.append((w.astype(np.float64), b.astype(np.float64)))
    assert off == params.size
    return out


def conv3x3(x, w, b):
    y = np.broadcast_to(b[None, :, None, None], (x.shape[0], w.shape[0]) + x.shape[2:]).copy()
    for ky in range(3):
        for kx in range(3):
            xs = np.roll(x, shift=(1 - ky, 1 - kx), axis=(2, 3))  # xs[y, x] = x[y + ky - 1, x + kx - 1]
            y += np.einsum("bchw,oc->bohw", xs, w[:, :, ky, kx])
    return y


def conv3x3_back(x, w, dy):
    dx = np.zeros_like(x)
    dw = np.zeros_like(w)
    for ky in range(3):
        for kx in range(3):
            xs = np.roll(x, shift=(1 - ky, 1 - kx), axis=(2, 3))
            dw[:, :, ky, kx] = np.einsum("bohw,bchw->oc", dy, xs)
            dx += np.roll(np.einsum("bohw,oc->bchw", dy, w[:, :, ky, kx]), shift=(ky - 1, kx - 1), axis=(2, 3))
    return dx, dw, dy.sum(axis=(0, 2, 3))


def gelu(z):
    return 0.5 * z * (1.0 + erf(z / np.sqrt(2.0)))


def gelu_grad(z):
    return 0.5 * (1.0 + erf(z / np.sqrt(2.0))) + z * np.exp(-0.5 * z * z) / np.sqrt(2.0 * np.pi)


def forward(params, layers, channels, x):
    x = x.astype(np.float64)
    cache = []
    a = x
    ps = unpack(params, layers, channels)
    for l, (w, b) in enumerate(ps):
        z = conv3x3(a, w, b)
        cache.append((a, z))
        a = gelu(z) if l + 1 < layers else z
    return a, cache


def loss_grad(params, layers, channels, x, t):
    y, cache = forward(params, layers, channels, x)
    t = t.astype(np.float64)
    n = y.size
    loss = float(np.sum((y - t) ** 2) / n)
    dz = 2.0 * (y - t) / n
    ps = unpack(params, layers, channels)
    grads = [None] * layers
    for l in range(layers - 1, -1, -1):
        a_in, z = cache[l]
        dx, dw, db = conv3x3_back(a_in, ps[l][0], dz)
        grads[l] = (dw, db)
        if l > 0:
            dz = dx * gelu_grad(cache[l - 1][1])
    g = np.concatenate([np.concatenate([dw.ravel(), db.ravel()]) for dw, db in grads])
    return loss, g
