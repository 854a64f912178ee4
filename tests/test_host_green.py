"""The Green's function the mixed solver's coarsest level uses (host code, no GPU): the
fast separable transform against the direct sum, and L g = delta - 1/N."""
import math

import numpy as np
import pytest

from maze_poisson_b200.c_api import CAPI


@pytest.fixture(scope="module")
def lib(product_path):
    return CAPI(product_path)


def direct(n):
    N = n ** 3
    w = 2 * math.pi / n
    k = np.arange(1, N)
    ki, kj, kk = k // (n * n), (k // n) % n, k % n
    lam = 2 * np.cos(w * ki) + 2 * np.cos(w * kj) + 2 * np.cos(w * kk) - 6.0
    d = np.arange(N)
    di, dj, dk = d // (n * n), (d // n) % n, d % n
    ph = np.cos(w * (np.outer(di, ki) + np.outer(dj, kj) + np.outer(dk, kk)))
    return ph @ (1.0 / lam) / N


@pytest.mark.parametrize("n", [4, 6, 10, 12, 16])
def test_green_function(lib, n):
    g = np.empty(n ** 3, dtype=np.float32)
    assert lib.mzb_coarse_green(n, g.ctypes.data) == 0
    if n <= 12:
        ref = direct(n)
        assert np.max(np.abs(g - ref)) <= 1e-6 * np.max(np.abs(ref))
    G = g.astype(np.float64).reshape(n, n, n)
    lap = sum(np.roll(G, s, a) for a in range(3) for s in (1, -1)) - 6 * G
    target = np.full((n, n, n), -1.0 / n ** 3)
    target[0, 0, 0] += 1.0
    assert np.max(np.abs(lap - target)) < 1e-6
    assert abs(G.sum()) < 1e-5 * np.max(np.abs(G)) * n ** 3  # zero mean: the constant mode is left out


def test_green_function_range(lib):
    g = np.empty(1, dtype=np.float32)
    assert lib.mzb_coarse_green(1, g.ctypes.data) == -1
    assert lib.mzb_coarse_green(17, g.ctypes.data) == -1
