"""Kernel-level parity of the CUDA path (through the C ABI's mzb_* entry points) against
the CPU oracle and the reference's golden vectors.

Bit-exact: every single sweep (Laplacian, RBGS, restriction, prolongation, CIC spread,
field-force interpolation, linked cells) -- the kernels keep the reference's per-point
operation order and round every product. Iterative solves agree to 1e-12 relative: only
the order of the global dot products differs (fixed, deterministic tree on the GPU).
"""
import os

import numpy as np
import pytest

from conftest import GOLDEN
from maze_poisson_b200.c_api import CAPI

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lib(product_path):
    c = CAPI(product_path)
    c.solver_initialize()
    return c


@pytest.fixture(scope="module")
def K():
    return np.load(os.path.join(GOLDEN, "kernels.npz"))


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def test_laplace_golden_bitexact(lib, K):
    out = np.empty((16, 16, 16))
    lib.mzb_laplace(np.ascontiguousarray(K["laplace_in"]), out, 16)
    assert np.array_equal(out, K["laplace_out"])


@pytest.mark.parametrize("n", [2, 3, 17, 48, 64, 96])
def test_laplace_sizes_bitexact(lib, oracle_lib, n):
    u = np.random.default_rng(n).standard_normal((n, n, n))
    a, b = np.empty_like(u), np.empty_like(u)
    lib.mzb_laplace(u, a, n)
    oracle_lib.orc_laplace(u, b, n)
    assert np.array_equal(a, b)


def test_rbgs_golden_bitexact(lib, K):
    x = np.ascontiguousarray(K["rbgs_x0"]).copy()
    lib.mzb_smooth_rbgs(np.ascontiguousarray(K["rbgs_rhs"]), x, 16, 3)
    assert np.array_equal(x, K["rbgs_out"])


def test_rbgs_64_bitexact(lib, oracle_lib):
    rng = np.random.default_rng(5)
    rhs, x0 = rng.standard_normal((2, 64, 64, 64))
    a, b = x0.copy(), x0.copy()
    lib.mzb_smooth_rbgs(np.ascontiguousarray(rhs), a, 64, 4)
    oracle_lib.orc_smooth_rbgs(np.ascontiguousarray(rhs), b, 64, 4)
    assert np.array_equal(a, b)


def test_restrict_prolong_golden_bitexact(lib, K):
    c = np.empty((8, 8, 8))
    lib.mzb_restrict27(np.ascontiguousarray(K["restrict_in"]), c, 16)
    assert np.array_equal(c, K["restrict_out"])
    f = np.empty((16, 16, 16))
    lib.mzb_prolong_trilinear(np.ascontiguousarray(K["prolong_in"]), f, 8)
    assert np.array_equal(f, K["prolong_out"])


def test_restrict_prolong_128_bitexact(lib, oracle_lib):
    rng = np.random.default_rng(9)
    f = rng.standard_normal((128, 128, 128))
    a, b = np.empty((64,) * 3), np.empty((64,) * 3)
    lib.mzb_restrict27(f, a, 128)
    oracle_lib.orc_restrict27(f, b, 128)
    assert np.array_equal(a, b)
    c = rng.standard_normal((64, 64, 64))
    fa, fb = np.empty((128,) * 3), np.empty((128,) * 3)
    lib.mzb_prolong_trilinear(c, fa, 64)
    oracle_lib.orc_prolong_trilinear(c, fb, 64)
    assert np.array_equal(fa, fb)


def test_conj_grad_golden(lib, K):
    b = np.ascontiguousarray(K["cg_b"])
    x = np.empty_like(b)
    it = lib.mzb_conj_grad(b, np.zeros_like(b), x, 1e-9, 16, 0)
    assert it == int(K["cg_iters"])
    assert rel(x, K["cg_x"]) < 1e-12


@pytest.mark.parametrize("precond", [0, 1])
def test_conj_grad_64(lib, oracle_lib, precond):
    rng = np.random.default_rng(11 + precond)
    xt = rng.standard_normal((64, 64, 64))
    b = np.empty_like(xt)
    oracle_lib.orc_laplace(xt, b, 64)
    x0 = 0.1 * rng.standard_normal((64, 64, 64))
    x = np.empty_like(b)
    it = lib.mzb_conj_grad(b, x0, x, 1e-8, 64, precond)
    assert it > 0
    # converged: |L x - b|_inf <= tol
    lx = np.empty_like(x)
    oracle_lib.orc_laplace(x, lx, 64)
    assert np.max(np.abs(lx - b)) <= 1e-8
    if precond == 0:
        xo = np.empty_like(b)
        ito = oracle_lib.orc_conj_grad(b, x0, xo, 1e-8, 64)
        assert abs(it - ito) <= 1
        assert rel(x, xo) < 1e-9


def test_cg_coarse_and_vcycle(lib, oracle_lib, K):
    xt = np.ascontiguousarray(K["mg_seed_x"])
    b = np.empty_like(xt)
    oracle_lib.orc_laplace(xt, b, 32)
    x = np.zeros_like(xt)
    lib.mzb_mg_apply(b, x, 32, 3)
    xo = np.zeros_like(xt)
    oracle_lib.orc_mg_apply(b, xo, 32, 3)
    assert rel(x, xo) < 1e-10
    bc = np.ascontiguousarray(b[::2, ::2, ::2])
    bc -= bc.mean()
    xc, xco = np.zeros_like(bc), np.zeros_like(bc)
    k1 = lib.mzb_cg_coarse(bc, xc, 16, 50, 1e-5)
    k2 = oracle_lib.orc_cg_coarse(bc, xco, 16, 50, 1e-5)
    assert k1 == k2
    assert rel(xc, xco) < 1e-10


@pytest.mark.parametrize("n", [32, 48, 64, 96, 128, 192, 256])
def test_fft_poisson_vs_numpy(lib, n):
    from oracle.fft_oracle import fft_poisson
    rng = np.random.default_rng(n)
    q = rng.standard_normal((n, n, n))
    q -= q.mean()
    L = 20.0
    phi = np.empty_like(q)
    lib.mzb_fft_poisson(q, phi, n, L, L / n)
    ref = fft_poisson(q, L, L / n)
    assert rel(phi, ref) < 1e-12


def test_ssor_golden_bitexact(lib):
    """The SSOR preconditioner's two wavefront solves equal the reference's serial ones."""
    g = np.load(os.path.join(GOLDEN, "ssor_kernels.npz"))
    for n in (2, 3, 4, 5, 6, 7, 8, 9, 16):
        x = np.ascontiguousarray(g[f"n{n}_in"])
        y = np.empty_like(x)
        lib.mzb_ssor_apply(x, y, n)
        assert np.array_equal(y, g[f"n{n}_out"]), n


@pytest.mark.parametrize("n", [31, 64])
def test_ssor_bitexact_vs_oracle(lib, oracle_lib, n):
    x = np.random.default_rng(n).standard_normal((n, n, n))
    a, b = np.empty_like(x), np.empty_like(x)
    lib.mzb_ssor_apply(x, a, n)
    oracle_lib.orc_ssor_apply(x, b, n)
    assert np.array_equal(a, b)


def test_conj_grad_ssor(lib, oracle_lib):
    """conj_grad_precond with SSOR (plcg.c:104-166): fewer iterations than the implicit
    Jacobi CG, converged to the absolute tolerance."""
    n = 32
    rng = np.random.default_rng(3)
    xt = rng.standard_normal((n, n, n))
    b = np.empty_like(xt)
    oracle_lib.orc_laplace(xt, b, n)
    x, x0 = np.empty_like(b), np.zeros_like(b)
    it = lib.mzb_conj_grad(b, x0, x, 1e-9, n, 3)
    it0 = lib.mzb_conj_grad(b, x0, np.empty_like(b), 1e-9, n, 0)
    assert 0 < it < it0
    lx = np.empty_like(x)
    oracle_lib.orc_laplace(x, lx, n)
    assert np.max(np.abs(lx - b)) <= 1e-9


@pytest.mark.parametrize("n", [10, 20, 40])
def test_blockjacobi_bitexact_vs_oracle(lib, oracle_lib, n):
    """The block-Jacobi product (precond_blockjacobi.c:173-206) with the same block inverse
    (Gauss-Jordan on the host, as the oracle computes it) and the reference's serial
    summation order is bit-exact; the oracle's inverse agrees with LAPACK's (numpy) to
    ~4e-15 relative (tests/test_oracle_pin.py)."""
    x = np.random.default_rng(n).standard_normal((n, n, n))
    a, b = np.empty_like(x), np.empty_like(x)
    lib.mzb_blockjacobi_apply(x, a, n)
    oracle_lib.orc_blockjacobi_apply(x, b, n)
    assert np.array_equal(a, b)


def test_conj_grad_blockjacobi(lib, oracle_lib):
    n = 20
    rng = np.random.default_rng(4)
    xt = rng.standard_normal((n, n, n))
    b = np.empty_like(xt)
    oracle_lib.orc_laplace(xt, b, n)
    x, x0 = np.empty_like(b), np.zeros_like(b)
    it = lib.mzb_conj_grad(b, x0, x, 1e-9, n, 4)
    assert it > 0
    lx = np.empty_like(x)
    oracle_lib.orc_laplace(x, lx, n)
    assert np.max(np.abs(lx - b)) <= 1e-9
