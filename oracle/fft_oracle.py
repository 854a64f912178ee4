"""Numpy restatement of the reference's FFT Poisson solve -- TEST INFRASTRUCTURE ONLY.

The reference computes, serially (library/src/fftw_wrap.c:166-189, plans at 142-163):
    X = r2c(q);  X[m] *= ig2[m] for every flat index m >= 1  (the DC term is skipped);
    phi = c2r(X)  (FFTW's unnormalised inverse; the 1/n^3 is folded into ig2)
with (library/src/grid_fft.c:89-120)
    ig2[i,j,k] = 4 pi / (h^3 n^3) / ((f_i^2 + f_j^2) + r_k^2 + 1e-10),  ig2[0] = 0,
    f = continuous wavenumbers 2 pi m / L (negative half from m = n/2 for even n),
    r = 2 pi k / L for k = 0..n/2.
The arithmetic lives in FFTW3, an external dependency the reference does not vendor
(found by CMake, library/CMakeLists.txt:37; no version pinned), absent in this image, so
this oracle is numpy.fft. Parity for this path is pinned only by these formulas: no
reference test or fixture exercises it.
"""
import numpy as np


def wavenumbers(n, L):
    nh = n // 2 + 1
    pi2 = 2 * np.pi
    m = np.arange(n, dtype=np.float64)
    first_neg = nh if n % 2 else nh - 1
    freq = np.where(np.arange(n) >= first_neg, pi2 * (m - n) / L, pi2 * m / L)
    rfreq = pi2 * np.arange(nh, dtype=np.float64) / L
    return freq, rfreq


def ig2(n, L, h):
    freq, rfreq = wavenumbers(n, L)
    const = 4 * np.pi / (h * h * h) / float(n * n * n)
    f1 = freq * freq
    f2 = f1[:, None] + (freq * freq)[None, :]
    g = const / (f2[:, :, None] + (rfreq * rfreq)[None, None, :] + 1e-10)
    g[0, 0, 0] = 0.0
    return g


def fft_poisson(q, L, h):
    """phi for the charge grid q (n^3), reference semantics (DC passed through)."""
    n = q.shape[0]
    X = np.fft.rfftn(q)
    g = ig2(n, L, h)
    dc = X[0, 0, 0]
    X = X * g
    X[0, 0, 0] = dc
    return np.fft.irfftn(X, s=q.shape, axes=(0, 1, 2)) * float(n * n * n)
