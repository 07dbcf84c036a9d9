"""CPU oracle for the learned-smoother network — TEST INFRASTRUCTURE ONLY.

Plain numpy restatement (float64) of the 3x3x3 convolution layers, their gradients, the masked
mean squared error and the Adam step that the library's CUDA kernels implement.  Only tests/
may import it, as the checker of those kernels.  The learned smoother has no counterpart in
the reference, so this oracle is pinned by a finite-difference check of its own gradients
(tests/test_learned_host.py) rather than by reference known answers.
"""
from __future__ import annotations

import numpy as np


def _pad(x):
    return np.pad(x, ((0, 0), (0, 0), (1, 1), (1, 1), (1, 1)))


def conv3d(x, w, b=None, relu=False):
    """x [B, Ci, Z, Y, X], w [Co, Ci, 27] (tap k = kx + 3 ky + 9 kz) -> y [B, Co, Z, Y, X]."""
    B, Ci, Z, Y, X = x.shape
    Co = w.shape[0]
    xp = _pad(np.asarray(x, dtype=np.float64))
    y = np.zeros((B, Co, Z, Y, X))
    for k in range(27):
        kx, ky, kz = k % 3, (k // 3) % 3, k // 9
        sl = xp[:, :, kz:kz + Z, ky:ky + Y, kx:kx + X]            # x[v + off(k)]
        y += np.einsum("oi,bizyx->bozyx", w[:, :, k], sl)
    if b is not None:
        y += np.asarray(b)[None, :, None, None, None]
    if relu:
        y = np.maximum(y, 0.0)
    return y


def conv3d_backward(x, w, gy):
    """(gx, gw, gb) of y = conv3d(x, w, b) for the output gradient gy."""
    B, Ci, Z, Y, X = x.shape
    xp = _pad(np.asarray(x, dtype=np.float64))
    gxp = np.zeros_like(xp)
    gw = np.zeros(w.shape)
    for k in range(27):
        kx, ky, kz = k % 3, (k // 3) % 3, k // 9
        sl = xp[:, :, kz:kz + Z, ky:ky + Y, kx:kx + X]
        gw[:, :, k] = np.einsum("bozyx,bizyx->oi", gy, sl)
        gxp[:, :, kz:kz + Z, ky:ky + Y, kx:kx + X] += np.einsum("oi,bozyx->bizyx", w[:, :, k], gy)
    gx = gxp[:, :, 1:-1, 1:-1, 1:-1]
    gb = gy.sum(axis=(0, 2, 3, 4))
    return gx, gw, gb


def mse(p, t, m=None, count=None):
    d = (p - t) * (1.0 if m is None else m)
    count = d.size if count is None else count
    return float(np.sum(d * d) / count), 2.0 * d / count


def adam(w, g, m, v, step, lr, b1=0.9, b2=0.999, eps=1e-8):
    m = b1 * m + (1 - b1) * g
    v = b2 * v + (1 - b2) * g * g
    w = w - lr * (m / (1 - b1 ** step)) / (np.sqrt(v / (1 - b2 ** step)) + eps)
    return w, m, v


class Net:
    """The smoother network: conv(ReLU) x 3 + conv, weights [(w, b)] per layer."""

    def __init__(self, layers):
        self.layers = layers

    def forward(self, x):
        acts = [x]
        for i, (w, b) in enumerate(self.layers):
            acts.append(conv3d(acts[-1], w, b, relu=i + 1 < len(self.layers)))
        return acts

    def gradients(self, x, target, mask=None, count=None):
        acts = self.forward(x)
        loss, g = mse(acts[-1], target, mask, count)
        grads = []
        for i in reversed(range(len(self.layers))):
            if i + 1 < len(self.layers):
                g = g * (acts[i + 1] > 0)
            gx, gw, gb = conv3d_backward(acts[i], self.layers[i][0], g)
            grads.append((gw, gb))
            g = gx
        return loss, list(reversed(grads))
