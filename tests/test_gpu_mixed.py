"""Multigrid field solve with FP64 refinement, in its two forms: mixed precision (FP32
V-cycles, precision 1) and FP64 multigrid (the same V-cycles in FP64, precision 2). Both
solve the same systems to the same FP64 residual tolerance as the reference's FP64
solvers, with a different inner algorithm. Checked against the CPU oracle's FP64 path
solved to the same tolerance; the bound is the one the mixed form is specified to meet,
force error below 1e-6 relative (max-norm ratio; much tighter in practice)."""
import ctypes

import numpy as np
import pytest

from maze_poisson_b200.c_api import CAPI
from maze_poisson_b200.md import MDRun
from maze_poisson_b200.systems import make_system

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


@pytest.fixture(scope="module")
def prod(product_path):
    return CAPI(product_path)


@pytest.fixture(scope="module")
def orc(oracle_path):
    return CAPI(oracle_path, extensions=False)


class MixedRun(MDRun):
    def __init__(self, *args, precision=1, plan=-1, sweeps=None, **kw):
        super().__init__(*args, precision=precision, **kw)
        self.plan = plan
        self.sweeps = sweeps

    def initialize(self):
        c = self.capi
        c.solver_initialize()
        maps = c.type_maps()
        s = self.sys
        c.solver_initialize_grid(s.n_grid, s.L, s.h, self.tol, self.eps_s, self.eps_int,
                                 maps["method"][self.method], maps["precond"][self.precond])
        c.mzb_set_precision(self.precision, 0.0)
        assert c.mzb_get_precision() == self.precision
        assert c.mzb_set_mixed_plan(self.plan) == 0
        if self.sweeps is not None:
            assert c.mzb_set_mixed_sweeps(*self.sweeps) == 0
        c.solver_initialize_particles(s.n_grid, 2, s.L, s.h, s.n_ions, maps["potential"]["TF"],
                                      maps["cas"]["CIC"], s.types, s.pos, s.vel, s.mass, s.charges,
                                      s.pot_params)
        c.solver_initialize_integrator(s.n_ions, self.dt, self.T, self.gamma,
                                       maps["integrator"][self.integrator], 1 if self.thermostat else 0)
        self.update_charges()
        c.solver_init_field()
        self.compute_forces()
        c.integrator_part_1()
        self.update_charges()
        c.solver_init_field()
        self.compute_forces()
        c.integrator_part_2()


@pytest.mark.parametrize("plan", [1, 0])
@pytest.mark.parametrize("precision", [1, 2])
@pytest.mark.parametrize("method", ["LCG", "MAZE-LCG", "MULTIGRID", "MAZE-MULTIGRID"])
def test_mixed_matches_fp64_oracle(prod, orc, method, precision, plan):
    """Coarse-level plan 1: the 32^3 coarse level solved by FFT; plan 0: levels down to 16^3,
    solved by the Green's function."""
    system = make_system(5, 64, seed=21)
    a = MixedRun(prod, system.copy(), method=method, tol=1e-10, precision=precision, plan=plan)
    b = MDRun(orc, system.copy(), method=method, tol=1e-10)
    a.initialize()
    b.initialize()
    assert prod.mzb_get_mixed_plan() == plan
    try:
        for step in range(3):
            sa, sb = a.state(), b.state()
            e_elec, e_tot = rel(sa["fcs_elec"], sb["fcs_elec"]), rel(sa["fcs_tot"], sb["fcs_tot"])
            print(f"{method} precision {precision} step {step}: fcs_elec {e_elec:.3e} fcs_tot {e_tot:.3e}")
            assert e_elec < 1e-7, (step, e_elec)
            assert e_tot < 1e-7, (step, e_tot)
            assert rel(sa["pos"], sb["pos"]) < 1e-10
            a.step()
            b.step()
            assert 0 <= a.n_iters < 30, a.n_iters
    finally:
        a.finalize()
        b.finalize()


@pytest.mark.parametrize("plan", [1, 2, 0])
@pytest.mark.parametrize("precision", [1, 2])
def test_mixed_solution_residual_meets_tol(prod, oracle_lib, precision, plan):
    """The returned field satisfies |L phi - b|_inf <= tol in FP64, with the 64^3 or the
    32^3 level solved by FFT, or the levels down to 16^3."""
    system = make_system(10, 128, density=1.329, seed=5)
    run = MixedRun(prod, system, method="LCG", tol=1e-9, precision=precision, plan=plan)
    run.initialize()
    assert prod.mzb_get_mixed_plan() == plan
    try:
        run.step()
        st = run.state()
        lphi = np.empty_like(st["field"])
        oracle_lib.orc_laplace(np.ascontiguousarray(st["field"]), lphi, 128)
        b = st["q"] * (-4 * np.pi / system.h)
        assert np.max(np.abs(lphi - b)) <= 1e-9 * 1.0001
    finally:
        run.finalize()


@pytest.mark.parametrize("sweeps", [None, (2, 2), (1, 1), (4, 3)])
def test_mixed_sweeps(prod, oracle_lib, sweeps):
    """Sweeps before / after the coarse correction (mzb_set_mixed_sweeps; V(3,2) unless
    set): every choice solves to the same FP64 tolerance, fewer sweeps taking more
    refinements; counts outside 1 .. 16 are refused."""
    system = make_system(10, 128, density=1.329, seed=5)
    run = MixedRun(prod, system, method="LCG", tol=1e-9, precision=1, sweeps=sweeps)
    run.initialize()
    try:
        nu1, nu2 = ctypes.c_int(), ctypes.c_int()
        prod.mzb_get_mixed_sweeps(ctypes.byref(nu1), ctypes.byref(nu2))
        assert (nu1.value, nu2.value) == (sweeps or (3, 2))
        for bad in ((0, 2), (2, 0), (17, 2), (2, 17)):
            assert prod.mzb_set_mixed_sweeps(*bad) == -1
        prod.mzb_get_mixed_sweeps(ctypes.byref(nu1), ctypes.byref(nu2))
        assert (nu1.value, nu2.value) == (sweeps or (3, 2))
        run.step()
        st = run.state()
        lphi = np.empty_like(st["field"])
        oracle_lib.orc_laplace(np.ascontiguousarray(st["field"]), lphi, 128)
        b = st["q"] * (-4 * np.pi / system.h)
        assert np.max(np.abs(lphi - b)) <= 1e-9 * 1.0001
        print(f"V{sweeps or (3, 2)}: {run.n_iters} refinements")
        assert 0 <= run.n_iters < (30 if sweeps == (1, 1) else 15)
    finally:
        run.finalize()


@pytest.mark.parametrize("method", ["LCG", "MAZE-LCG", "MULTIGRID", "MAZE-MULTIGRID"])
def test_fp16_level0_programs_256(prod, oracle_lib, method):
    """At 256^3 the FP32+refine form stores level 0 as FP16 (scaled by the residual's max):
    every program that takes it (the LCG and MaZe updates, the multigrid updates from the
    extrapolated start) still returns a field with |L phi - b|_inf within the FP64 tol."""
    system = make_system(4, 256, density=1.379, seed=9)
    run = MixedRun(prod, system, method=method, tol=1e-9, precision=1)
    run.initialize()
    try:
        for _ in range(2):
            run.step()
            assert 0 <= run.n_iters < 30, run.n_iters
        st = run.state()
        lphi = np.empty_like(st["field"])
        oracle_lib.orc_laplace(np.ascontiguousarray(st["field"]), lphi, 256)
        b = st["q"] * (-4 * np.pi / system.h)
        assert np.max(np.abs(lphi - b)) <= 1e-9 * 1.0001
    finally:
        run.finalize()


def test_fp16_level0_scale_guard(prod, oracle_lib):
    """The FP16 level 0 starts in the units of the grid's last first residual. A start far
    from the solution (the field plus noise of 1e3) and then one very close to it (noise of
    1e-6) each leave the range those units cover: the residual is written again in its own
    units, and both solves meet the FP64 tol."""
    system = make_system(4, 256, density=1.379, seed=11)
    run = MixedRun(prod, system, method="LCG", tol=1e-9, precision=1)
    run.initialize()
    try:
        n = 256
        st = run.state()
        phi = np.ascontiguousarray(st["field"])
        b = st["q"] * (-4 * np.pi / system.h)
        rng = np.random.default_rng(3)
        for amp in (1e3, 1e-6):
            prod.solver_set_field(np.ascontiguousarray(phi + amp * rng.standard_normal(phi.shape)))
            res = prod.solver_update_field()
            assert 0 <= res < 30, (amp, res)
            prod.get_field(phi)
            lphi = np.empty_like(phi)
            oracle_lib.orc_laplace(phi, lphi, n)
            assert np.max(np.abs(lphi - b)) <= 1e-9 * 1.0001, amp
    finally:
        run.finalize()


@pytest.mark.parametrize("plan", [2, 0])
def test_fp16_level0_plans_256(prod, oracle_lib, plan):
    """FP16 level 0 at 256^3 under the other coarse-level plans: the 128^3 level swept in
    FP32 and the 64^3 level solved by FFT (plan 2), or the levels down to 16^3 solved by
    the Green's function (plan 0); the field meets the FP64 tol."""
    system = make_system(4, 256, density=1.379, seed=13)
    run = MixedRun(prod, system, method="LCG", tol=1e-9, precision=1, plan=plan)
    run.initialize()
    assert prod.mzb_get_mixed_plan() == plan
    try:
        run.step()
        assert 0 <= run.n_iters < 30, run.n_iters
        st = run.state()
        lphi = np.empty_like(st["field"])
        oracle_lib.orc_laplace(np.ascontiguousarray(st["field"]), lphi, 256)
        b = st["q"] * (-4 * np.pi / system.h)
        assert np.max(np.abs(lphi - b)) <= 1e-9 * 1.0001
    finally:
        run.finalize()
