"""Seeded Gaussian random fields for variable diffusion coefficients a = exp(g).

g has mean 0 and the squared-exponential covariance C(r) = variance * exp(-r^2 / (2 l^2)).
It is sampled exactly (up to the grid) by circulant embedding: on a periodic grid that covers
the domain plus a margin of several correlation lengths, the covariance matrix is circulant,
its eigenvalues are the FFT of its first row, and g = IFFT(sqrt(lambda) * FFT(w)) for white
noise w has exactly that covariance (C. R. Dietrich and G. N. Newsam, SIAM J. Sci. Comput. 18
(1997) 1088-1107).  Values between grid points come from trilinear interpolation.
"""
from __future__ import annotations

import numpy as np


class GaussianRandomField:
    def __init__(self, seed, corr_length=0.05, variance=2.0, origin=(0.0, 0.0, 0.0), extent=(1.0, 1.0, 1.0),
                 points_per_length=4.0, margin=4.0):
        self.corr_length = float(corr_length)
        self.variance = float(variance)
        self.origin = np.asarray(origin, dtype=np.float64)
        D = len(self.origin)
        ext = np.asarray(extent, dtype=np.float64)
        h = self.corr_length / points_per_length
        pad = margin * self.corr_length
        n = [int(np.ceil((e + pad) / h)) for e in ext]
        n = [m + (m % 2) for m in n]
        self.h = h
        self.n = n
        # periodic distance of every grid point to the origin point
        axes = [np.minimum(np.arange(m), m - np.arange(m)) * h for m in n]
        grids = np.meshgrid(*axes, indexing="ij")
        r2 = sum(g * g for g in grids)
        c = self.variance * np.exp(-r2 / (2.0 * self.corr_length ** 2))
        lam = np.fft.fftn(c).real
        lam = np.maximum(lam, 0.0)
        rng = np.random.default_rng(seed)
        w = rng.standard_normal(n)
        self.values = np.fft.ifftn(np.sqrt(lam) * np.fft.fftn(w)).real   # [n0, n1, n2]
        self.D = D

    def __call__(self, X):
        """g at physical points X [m, D] (trilinear interpolation)."""
        X = np.atleast_2d(np.asarray(X, dtype=np.float64))
        t = (X - self.origin[None, :]) / self.h
        i0 = np.floor(t).astype(np.int64)
        f = t - i0
        out = np.zeros(X.shape[0])
        for corner in range(1 << self.D):
            idx = []
            wgt = np.ones(X.shape[0])
            for a in range(self.D):
                bit = (corner >> a) & 1
                idx.append(np.clip(i0[:, a] + bit, 0, self.n[a] - 1))
                wgt = wgt * (f[:, a] if bit else 1.0 - f[:, a])
            out += wgt * self.values[tuple(idx)]
        return out

    def coefficient(self):
        """a(x) = exp(g(x)) as a VariableDiffusion coefficient callable."""
        return lambda X: np.exp(self(X))
