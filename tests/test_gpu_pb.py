"""Poisson-Boltzmann parity of the CUDA path against the CPU oracle (which the golden
vectors under tests/golden pin bit for bit to the reference's own PB code), through the
C ABI.

Tolerances:
  * bit-exact: the PB operator, one PB smoother iteration, the coarse coefficient
    restrictions -- each keeps the reference's per-point order and rounds every product;
  * face coefficients and screening after solver_update_eps_k2: 1e-14 relative. The
    factors of overlapping solvation shells are multiplied in ion order as the reference
    does; only the cube differs (correctly rounded here, glibc's pow(x, 3) is one ulp off
    in ~0.08 % of inputs);
  * PB solves (CG, V-cycle): 1e-10 relative, CG iterations within 1 (dot-product order);
  * boundary forces: 1e-11 of the largest component of the same array (a fixed-tree sum
    over each ion's box in place of the reference's serial loop);
  * MD: 1e-10 relative per step, as for the Poisson grids.
"""
import os

import numpy as np
import pytest

from conftest import GOLDEN
from maze_poisson_b200.c_api import CAPI
from maze_poisson_b200.md import MDRun
from maze_poisson_b200.systems import make_pb_system, make_system, pb_settings

pytestmark = pytest.mark.gpu
TOL = 1e-10


def rel(a, b):
    a, b = np.asarray(a, dtype=np.float64), np.asarray(b, dtype=np.float64)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def pb_inputs(n, seed):
    """The seeded PB kernel inputs of tests/golden/make_golden.py."""
    rng = np.random.default_rng(seed)
    ex, ey, ez = (1.0 + 77.0 * rng.random((n, n, n)) for _ in range(3))
    k2 = 0.05 * rng.random((n, n, n))
    xt = rng.standard_normal((n, n, n))
    return ex, ey, ez, k2, xt


@pytest.fixture(scope="module")
def lib(product_path):
    c = CAPI(product_path)
    c.solver_initialize()
    return c


@pytest.fixture(scope="module")
def PBK():
    return np.load(os.path.join(GOLDEN, "pb_kernels.npz"))


def test_pb_sweeps_golden_bitexact(lib, PBK):
    n = 16
    ex, ey, ez, k2, xt = pb_inputs(n, int(PBK["n16_seed"]))
    b = np.empty_like(xt)
    lib.mzb_laplace_pb(xt, b, ex, ey, ez, k2, n)
    assert np.array_equal(b, PBK["n16_b"])
    rng = np.random.default_rng(99)
    rhs = rng.standard_normal((n, n, n))
    x = rng.standard_normal((n, n, n))
    lib.mzb_smooth_pb(rhs, x, n, 3, ex, ey, ez, k2)
    assert np.array_equal(x, PBK["rbgs_out"])
    c = [np.empty((8, 8, 8)) for _ in range(4)]
    lib.mzb_restrict_pb(ex, ey, ez, k2, *c, n)
    for arr, name in zip(c, ("ex", "ey", "ez", "k2")):
        assert np.array_equal(arr, PBK[f"restrict_{name}"]), name


def test_pb_sweeps_64_bitexact(lib, oracle_lib):
    n = 64
    ex, ey, ez, k2, xt = pb_inputs(n, 77)
    a, b = np.empty_like(xt), np.empty_like(xt)
    lib.mzb_laplace_pb(xt, a, ex, ey, ez, k2, n)
    oracle_lib.orc_laplace_pb(xt, b, ex, ey, ez, k2, n)
    assert np.array_equal(a, b)
    rhs = np.ascontiguousarray(xt[::-1])
    xa, xb = np.zeros_like(xt), np.zeros_like(xt)
    lib.mzb_smooth_pb(rhs, xa, n, 2, ex, ey, ez, k2)
    oracle_lib.orc_smooth_pb(rhs, xb, n, 2, ex, ey, ez, k2)
    assert np.array_equal(xa, xb)


def test_pb_cg_and_vcycle(lib, oracle_lib, PBK):
    n = 16
    ex, ey, ez, k2, xt = pb_inputs(n, int(PBK["n16_seed"]))
    b = np.ascontiguousarray(PBK["n16_b"])
    x = np.empty_like(b)
    it = lib.mzb_conj_grad_pb(b, np.zeros_like(b), x, 1e-9, n, ex, ey, ez, k2)
    assert abs(it - int(PBK["cg_iters"])) <= 1
    assert rel(x, PBK["cg_x"]) < TOL
    n = 32
    ex, ey, ez, k2, xt = pb_inputs(n, int(PBK["n32_seed"]))
    b = np.empty_like(xt)
    oracle_lib.orc_laplace_pb(xt, b, ex, ey, ez, k2, n)
    xa, xb = np.zeros_like(xt), np.zeros_like(xt)
    lib.mzb_mg_pb_apply(b, xa, n, 4, ex, ey, ez, k2)
    oracle_lib.orc_mg_pb_apply(b, xb, n, 4, ex, ey, ez, k2)
    assert rel(xa, xb) < TOL
    assert np.array_equal(xb.reshape(-1)[::997], PBK["mg_x_sample"])


def setup_pb(capi, system, pb, method=0, eps_s=78.4):
    """The reference's PB set-up calls (solver.py:140-163, 346-356) without a solve."""
    c = capi
    c.solver_initialize()
    c.solver_initialize_grid(system.n_grid, system.L, system.h, 1e-10, eps_s, 1.0, method, 0)
    c.solver_initialize_grid_pois_boltz(pb.w, pb.kbar2, int(pb.nonpolar))
    c.solver_initialize_particles(system.n_grid, 2, system.L, system.h, system.n_ions, 0, 0, system.types,
                                  system.pos, system.vel, system.mass, system.charges, system.pot_params)
    c.solver_initialize_particles_pois_boltz(pb.gamma_np, pb.beta_np, pb.radii)
    c.solver_update_charges()
    c.solver_update_eps_k2()


@pytest.mark.parametrize("case", ["cluster", "melt686"])
def test_pb_coefficients_and_forces(product_path, oracle_path, oracle_lib, case):
    """eps/k2 after solver_update_eps_k2 and the boundary forces for one field. melt686:
    a dense melt (686 ions, more than one 512-ion candidate chunk per tile) where every
    point sits in many overlapping shells."""
    if case == "cluster":
        system = make_pb_system(8, 32, 16.0, seed=3)
    else:
        system = make_system(7, 32, density=1.379, T=300.0, seed=5)
    pb = pb_settings(system)
    prod, orc = CAPI(product_path), CAPI(oracle_path, extensions=False)
    setup_pb(prod, system, pb)
    setup_pb(orc, system, pb)
    try:
        g = system.n_grid
        a = [np.empty((g, g, g)) for _ in range(4)]
        b = [np.empty((g, g, g)) for _ in range(4)]
        prod.mzb_get_pb_grids(*a)
        oracle_lib.orc_get_pb_grids(*b)
        for x, y, name in zip(a, b, ("eps_x", "eps_y", "eps_z", "k2")):
            assert rel(x, y) < 1e-14, (name, rel(x, y))
            assert np.mean(x == y) > 0.99, name
        assert np.max(b[3]) > np.min(b[3])  # the screening term varies over the grid
        phi = np.random.default_rng(8).standard_normal((g, g, g))
        for c in (prod, orc):
            c.solver_set_field(phi)
            assert c.solver_compute_forces_pb() == 0.0
        radii = np.empty(system.n_ions)
        prod.get_radii(radii)
        assert np.array_equal(radii, pb.radii)
        for name in ("fcs_db", "fcs_ib", "fcs_np"):
            fa, fb = np.empty((system.n_ions, 3)), np.empty((system.n_ions, 3))
            getattr(prod, "get_" + name)(fa)
            getattr(orc, "get_" + name)(fb)
            assert np.max(np.abs(fb)) > 0, name
            assert rel(fa, fb) < 1e-11, (name, rel(fa, fb))
    finally:
        prod.solver_finalize()
        orc.solver_finalize()


def pb_pair(prod, orc, method, steps=2, nonpolar=1):
    system = make_pb_system(8, 32, 16.0, seed=3)
    pb = pb_settings(system, nonpolar=nonpolar)
    kw = dict(method=method, tol=1e-10 if "LCG" in method else 1e-8, integrator="VERLET", T=300.0,
              eps_s=78.4, eps_int=1.0, pb=pb)
    a, b = MDRun(prod, system.copy(), **kw), MDRun(orc, system.copy(), **kw)
    a.initialize()
    b.initialize()
    keys = ("field", "fcs_elec", "fcs_noel", "fcs_db", "fcs_ib", "fcs_np", "fcs_tot", "pos", "vel")
    try:
        for s in range(-1, steps):
            if s >= 0:
                a.step()
                b.step()
                assert abs(a.n_iters - b.n_iters) <= 1, (s, a.n_iters, b.n_iters)
            sa, sb = a.state(), b.state()
            for key in keys:
                assert rel(sa[key], sb[key]) < TOL, (s, key, rel(sa[key], sb[key]))
    finally:
        a.finalize()
        b.finalize()


@pytest.mark.parametrize("method", ["LCG", "MAZE-LCG", "MULTIGRID", "MAZE-MULTIGRID"])
def test_pb_md(product_path, oracle_path, method):
    pb_pair(CAPI(product_path), CAPI(oracle_path, extensions=False), method)


def test_pb_md_step_matches_per_call(product_path):
    """solver_md_step on a PB grid makes the reference's per-step calls (solver.py:483-492)."""
    prod = CAPI(product_path)
    out = []
    for native in (False, True):
        system = make_pb_system(8, 32, 16.0, seed=3)
        run = MDRun(prod, system, method="MAZE-LCG", tol=1e-10, integrator="VERLET", T=300.0,
                    eps_s=78.4, eps_int=1.0, pb=pb_settings(system))
        run.initialize()
        if native:
            prod.solver_md_step(2)
        else:
            run.step()
            run.step()
        out.append(run.state(fields=False))
        run.finalize()
    for key in ("pos", "vel", "fcs_tot"):
        assert np.array_equal(out[0][key], out[1][key]), key
