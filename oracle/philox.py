"""Numpy restatement of the O-block noise generator -- TEST INFRASTRUCTURE ONLY.

The reference's O-block draws N(0,1) variates from glibc rand() through a polar
Box-Muller with static state (library/src/integrator_ovrvo.c:12-36), which cannot be
reproduced off the reference's host. The B200 build uses counter-based Philox4x32-10
(Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy as 1, 2, 3", SC 2011)
so every draw is a pure function of (seed, O-block call, ion, component):

    counter = (ion, draw, call_lo, call_hi), key = (seed_lo, seed_hi), draw in {0, 1}
    u = ((hi << 32 | lo) >> 11 + 0.5) * 2^-53 for the word pairs (x0, x1) and (x2, x3)
    z0 = sqrt(-2 ln u1) cos(2 pi u2), z1 = sqrt(-2 ln u1) sin(2 pi u2)
    components (0, 1, 2) = (z0 of draw 0, z1 of draw 0, z0 of draw 1).

This restatement checks the GPU generator word for word (the uint32 outputs) and its
normals to within libm rounding.
"""
import numpy as np

M0 = np.uint64(0xD2511F53)
M1 = np.uint64(0xCD9E8D57)
W0 = np.uint32(0x9E3779B9)
W1 = np.uint32(0xBB67AE85)
MASK = np.uint64(0xFFFFFFFF)


def philox4x32_10(c0, c1, c2, c3, k0, k1):
    """Vectorised Philox4x32-10 on uint32 arrays; returns the four output words."""
    c0, c1, c2, c3 = (np.asarray(x, dtype=np.uint32) for x in (c0, c1, c2, c3))
    k0 = np.uint32(k0)
    k1 = np.uint32(k1)
    with np.errstate(over="ignore"):
        for _ in range(10):
            p0 = M0 * c0.astype(np.uint64)
            p1 = M1 * c2.astype(np.uint64)
            hi0, lo0 = (p0 >> np.uint64(32)).astype(np.uint32), (p0 & MASK).astype(np.uint32)
            hi1, lo1 = (p1 >> np.uint64(32)).astype(np.uint32), (p1 & MASK).astype(np.uint32)
            c0, c1, c2, c3 = hi1 ^ c1 ^ k0, lo1, hi0 ^ c3 ^ k1, lo0
            k0 = np.uint32(k0 + W0)
            k1 = np.uint32(k1 + W1)
    return c0, c1, c2, c3


def _u53(hi, lo):
    a = (hi.astype(np.uint64) << np.uint64(32)) | lo.astype(np.uint64)
    return ((a >> np.uint64(11)).astype(np.float64) + 0.5) * 2.0 ** -53


def normals(seed, call, n_ions):
    """(n_ions, 3) standard normals of O-block call `call`."""
    ion = np.arange(n_ions, dtype=np.uint32)
    out = np.empty((n_ions, 3))
    k0, k1 = seed & 0xFFFFFFFF, (seed >> 32) & 0xFFFFFFFF
    for draw in (0, 1):
        w = philox4x32_10(ion, np.full(n_ions, draw, np.uint32),
                          np.full(n_ions, call & 0xFFFFFFFF, np.uint32),
                          np.full(n_ions, (call >> 32) & 0xFFFFFFFF, np.uint32), k0, k1)
        u1, u2 = _u53(w[0], w[1]), _u53(w[2], w[3])
        rad = np.sqrt(-2.0 * np.log(u1))
        out[:, 2 * draw] = rad * np.cos(2 * np.pi * u2)
        if draw == 0:
            out[:, 1] = rad * np.sin(2 * np.pi * u2)
    return out
