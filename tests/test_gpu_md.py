"""MD-level parity of the CUDA path against the CPU oracle, through the reference's C ABI.

Both libraries are driven by the same MDRun call sequence (the reference's SolverMD).
Tolerances (FP64 mode):
  * bit-exact: CIC corner indices, the charge grid q and the field force for the same
    positions and phi, linked cells;
  * 1e-10 relative (max-norm ratio): fields, forces, energies, positions and velocities
    after each step -- the only differences come from the dot-product order inside the
    iterative solves and from exp/pow in the pair forces.
"""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

import mdparity
from conftest import GOLDEN, ROOT
from maze_poisson_b200.c_api import CAPI
from maze_poisson_b200.md import MDRun
from maze_poisson_b200.systems import make_system, pair_system

pytestmark = pytest.mark.gpu
TOL = 1e-10
rel = mdparity.rel


@pytest.fixture(scope="module")
def prod(product_path):
    return CAPI(product_path)


@pytest.fixture(scope="module")
def orc(oracle_path):
    return CAPI(oracle_path, extensions=False)


def run_pair(prod, orc, system, steps, check_each=True, noise=False, **kw):
    return mdparity.run_pair(prod, orc, system, steps, check_each=check_each, noise=noise, bound=TOL, **kw)[:2]


SCEN = json.load(open(os.path.join(GOLDEN, "scenarios.json")))


@pytest.mark.parametrize("name", sorted(SCEN))
def test_golden_scenarios(prod, name):
    """Product against the reference's own trajectories (tests/golden)."""
    ncell, ng, method, precond, tol, itg, thermo, steps = SCEN[name][:8]
    cas = SCEN[name][8] if len(SCEN[name]) > 8 else "CIC"
    pot = SCEN[name][9] if len(SCEN[name]) > 9 else "TF"
    g = np.load(os.path.join(GOLDEN, f"md_{name}.npz"))
    system = pair_system(ncell, ng, pot, density=1.379, T=1200.0, seed=7)
    run = MDRun(prod, system, method=method, precond=precond, tol=tol, integrator=itg,
                thermostat=thermo, cas=cas, pot=pot)
    run.initialize()
    try:
        st = run.state()
        for key in ("fcs_tot", "fcs_elec", "fcs_noel", "pos", "vel"):
            assert rel(st[key], g["init_" + key]) < TOL, key
        if "init_q" in g:
            if cas == "SPL_CUBIC":  # the GPU's correctly rounded cube vs glibc pow(x, 3): <= 1 ulp
                assert rel(st["q"], g["init_q"]) < 1e-14
            else:
                assert np.array_equal(st["q"], g["init_q"])
        for s in range(steps):
            run.step()
            st = run.state()
            assert abs(st["n_iters"] - int(g[f"s{s}_iters"])) <= 1
            for key in ("pos", "vel", "fcs_tot"):
                assert rel(st[key], g[f"s{s}_{key}"]) < TOL, (s, key)
            assert rel(st["field"].reshape(-1)[::101], g[f"s{s}_field_sample"]) < TOL
    finally:
        run.finalize()


def test_lcg_verlet_250(prod, orc):
    run_pair(prod, orc, make_system(5, 64, seed=3), 6, method="LCG", tol=1e-7)


def test_maze_lcg_250(prod, orc):
    run_pair(prod, orc, make_system(5, 64, seed=4), 4, method="MAZE-LCG", tol=1e-7)


def test_maze_lcg_jacobi_250(prod, orc):
    run_pair(prod, orc, make_system(5, 64, seed=5), 3, method="MAZE-LCG", precond="JACOBI", tol=1e-7)


def test_multigrid_250(prod, orc):
    run_pair(prod, orc, make_system(5, 64, seed=6), 2, method="MULTIGRID", tol=1e-7)


def test_maze_multigrid_250(prod, orc):
    run_pair(prod, orc, make_system(5, 64, seed=8), 2, method="MAZE-MULTIGRID", tol=1e-7)


def test_ovrvo_thermostat_injected_noise(prod, orc):
    """OVRVO with the thermostat on: the oracle's O-block is fed the GPU's Philox draws."""
    run_pair(prod, orc, make_system(3, 32, seed=9), 4, noise=True, method="LCG", tol=1e-9,
             integrator="OVRVO", thermostat=True, gamma_per_ps=1.0)


def test_fft_path(prod, oracle_lib):
    """FFT method: q bit-exact, phi = numpy oracle of the same q, forces bit-exact."""
    from oracle.fft_oracle import fft_poisson
    system = make_system(5, 64, seed=10)
    run = MDRun(prod, system.copy(), method="FFT")
    run.initialize()
    try:
        for _ in range(2):
            run.step()
        st = run.state()
        s = run.sys
        assert rel(st["field"], fft_poisson(st["q"], s.L, s.h)) < 1e-12
        # the last forces were computed from the current positions (part 2 only kicks)
        nbr = np.empty((s.n_ions, 8, 3), dtype=np.int64)
        oracle_lib.orc_cic_neighbors(st["pos"], s.n_ions, s.n_grid, s.h, nbr)
        f = np.empty((s.n_ions, 3))
        oracle_lib.orc_force_fd(st["field"], nbr, s.charges, st["pos"], s.n_ions, s.n_grid, s.h, f)
        assert np.array_equal(st["fcs_elec"], f)
        # FFT keeps no previous field: get_field_prev returns phi (solver_md.c:289-292)
        assert np.array_equal(st["field_prev"], st["field"])
    finally:
        run.finalize()


def test_particle_kernels_bitexact(prod, oracle_lib):
    """CIC corners, q, field force of a given phi, linked cells, and the Tosi-Fumi forces."""
    s = make_system(10, 64, density=1.329, seed=12)
    # exercise the box edges: ions at 0, at L - tiny, and a dense cluster in one tile
    s.pos[0] = [0.0, 0.0, 0.0]
    s.pos[1] = [s.L * (1 - 1e-16), s.L * 0.5, s.L * (1 - 1e-15)]
    s.pos[2:40] = s.pos[2] * 0 + np.array([1.0, 1.0, 1.0]) * s.h * 0.25 + \
        np.random.default_rng(0).uniform(0, s.h * 3.5, (38, 3))
    run = MDRun(prod, s, method="LCG", tol=1e-6)
    prod.solver_initialize()
    maps = prod.type_maps()
    prod.solver_initialize_grid(s.n_grid, s.L, s.h, 1e-6, 1.0, 1.0, maps["method"]["LCG"], 0)
    prod.solver_initialize_particles(s.n_grid, 2, s.L, s.h, s.n_ions, 0, 0, s.types, s.pos, s.vel,
                                     s.mass, s.charges, s.pot_params)
    prod.solver_initialize_integrator(s.n_ions, 1.0, 1200.0, 0.0, 1, 0)
    try:
        # charges: 38 clustered ions make the grid non-neutral locally but the total stays 0
        assert prod.solver_update_charges() == 0
        nbr = np.empty((s.n_ions, 8, 3), dtype=np.int64)
        prod.mzb_get_cic_neighbors(nbr)
        nbo = np.empty_like(nbr)
        oracle_lib.orc_cic_neighbors(s.pos, s.n_ions, s.n_grid, s.h, nbo)
        assert np.array_equal(nbr, nbo)
        q = np.empty((64, 64, 64))
        prod.get_q(q)
        qo = np.empty_like(q)
        oracle_lib.orc_spread_cic(s.pos, s.charges, nbo, s.n_ions, 64, s.h, qo)
        assert np.array_equal(q, qo)
        # field force on an arbitrary phi
        phi = np.random.default_rng(1).standard_normal((64, 64, 64))
        prod.solver_set_field(phi)
        prod.solver_compute_forces_elec()
        fe = np.empty((s.n_ions, 3))
        prod.get_fcs_elec(fe)
        feo = np.empty_like(fe)
        oracle_lib.orc_force_fd(phi, nbo, s.charges, s.pos, s.n_ions, 64, s.h, feo)
        assert np.array_equal(fe, feo)
        # linked cells
        for nc in (3, 4, 7):
            prod.mzb_set_cell_grid(nc)
            st = np.empty(nc ** 3 + 1, dtype=np.int32)
            io = np.empty(s.n_ions, dtype=np.int32)
            assert prod.mzb_get_cells(st, io) == nc
            sto, ioo = np.empty_like(st), np.empty_like(io)
            oracle_lib.orc_cell_list(s.pos, s.n_ions, s.L, nc, sto, ioo)
            assert np.array_equal(st, sto) and np.array_equal(io, ioo)
        # Tosi-Fumi forces and energy
        tab = np.empty(28)
        oracle_lib.orc_tf_table(s.pot_params, 2, s.L, tab)
        for nc in (1, 4):
            prod.mzb_set_cell_grid(nc)
            e = prod.solver_compute_forces_noel()
            fn = np.empty((s.n_ions, 3))
            prod.get_fcs_noel(fn)
            fno = np.empty_like(fn)
            eo = oracle_lib.orc_tf_forces(s.pos, s.types, tab, 2, s.n_ions, s.L, s.L / 2, fno)
            assert rel(fn, fno) < 1e-12
            assert abs(e - eo) < 1e-10 * abs(eo)
    finally:
        prod.solver_finalize()


def test_philox_matches_restatement(prod):
    from oracle.philox import normals
    s = make_system(3, 32, seed=1)
    run = MDRun(prod, s, integrator="OVRVO", thermostat=True)
    prod.solver_initialize()
    prod.solver_initialize_grid(32, s.L, s.h, 1e-7, 1.0, 1.0, 0, 0)
    prod.solver_initialize_particles(32, 2, s.L, s.h, s.n_ions, 0, 0, s.types, s.pos, s.vel, s.mass,
                                     s.charges, s.pot_params)
    try:
        for seed, call in [(0x5eed, 0), (0x5eed, 7), (2 ** 40 + 3, 2 ** 33 + 1)]:
            prod.mzb_set_seed(seed)
            z = np.empty((s.n_ions, 3))
            prod.mzb_philox_normals(call, z)
            assert np.max(np.abs(z - normals(seed, call, s.n_ions))) < 1e-13
        prod.mzb_set_seed(0x5eed)
    finally:
        prod.solver_finalize()
    del run


def test_charge_conservation_failure_exits():
    """A non-neutral system makes solver_update_charges print and exit(1), as the
    reference does (library/src/solver_md.c:91-107)."""
    code = f"""
import sys; sys.path.insert(0, {ROOT!r})
import numpy as np
from maze_poisson_b200.c_api import CAPI
from maze_poisson_b200.systems import make_system, pair_system
s = make_system(2, 16, seed=1)
s.charges[0] = 3.0
c = CAPI(); c.solver_initialize()
c.solver_initialize_grid(16, s.L, s.h, 1e-7, 1.0, 1.0, 0, 0)
c.solver_initialize_particles(16, 2, s.L, s.h, s.n_ions, 0, 0, s.types, s.pos, s.vel, s.mass, s.charges, s.pot_params)
c.solver_update_charges()
print("not reached")
"""
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=300,
                       env=dict(os.environ, MZB_QUIET="1"))
    assert r.returncode == 1
    assert "Charge conservation error" in r.stdout
    assert "not reached" not in r.stdout


def test_charge_conservation_failure_exits_in_md_step():
    """solver_md_step keeps the charge check on the device and reads it after the steps;
    a non-neutral system still prints the reference's message and exits 1."""
    code = f"""
import sys; sys.path.insert(0, {ROOT!r})
from maze_poisson_b200.c_api import CAPI
from maze_poisson_b200.systems import make_system
s = make_system(2, 16, seed=1)
s.charges[0] = 3.0
c = CAPI(); c.solver_initialize()
c.solver_initialize_grid(16, s.L, s.h, 1e-7, 1.0, 1.0, 0, 0)
c.solver_initialize_particles(16, 2, s.L, s.h, s.n_ions, 0, 0, s.types, s.pos, s.vel, s.mass, s.charges, s.pot_params)
c.solver_initialize_integrator(s.n_ions, 40.0, 1200.0, 0.0, 1, 0)
c.solver_md_step(3)
print("not reached")
"""
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=300,
                       env=dict(os.environ, MZB_QUIET="1"))
    assert r.returncode == 1, (r.returncode, r.stdout, r.stderr[-2000:])
    assert "Charge conservation error: q_tot = 0.000000, q_tot_loc = 2.000000" in r.stdout
    assert "not reached" not in r.stdout


def test_md_step_matches_per_call_sequence(prod):
    """solver_md_step(n) (device-side checks, one synchronisation) gives the same state as
    the reference's per-call sequence, FP64 and mixed forms."""
    for precision in (0, 1):
        out = []
        for batched in (False, True):
            run = MDRun(prod, make_system(5, 64, seed=3), method="LCG", tol=1e-9, precision=precision)
            run.initialize()
            try:
                if batched:
                    res = prod.solver_md_step(4)
                else:
                    for _ in range(4):
                        res = run.step()
                st = run.state()
                st["res"] = res
                out.append(st)
            finally:
                run.finalize()
        a, b = out
        assert a["res"] == b["res"]
        for key in ("field", "field_prev", "q", "fcs_tot", "pos", "vel"):
            assert np.array_equal(a[key], b[key]), (precision, key)


@pytest.mark.parametrize("cas", ["SPL_QUADR", "SPL_CUBIC"])
def test_spline_kernels(prod, oracle_lib, cas):
    """B-spline charge assignment (charges.c:16-38, particles.c:348-385): the 64-point
    neighbour lists are equal; q and the field force of a given phi are bit-exact for the
    quadratic spline and within 1e-14 for the cubic one (the GPU's correctly rounded cube
    vs glibc pow(x, 3), which is one ulp off in ~0.08 % of inputs)."""
    code = {"SPL_QUADR": 1, "SPL_CUBIC": 2}[cas]
    s = make_system(10, 64, density=1.329, seed=31)
    s.pos[0] = [0.0, 0.0, 0.0]
    s.pos[1] = [s.L * (1 - 1e-16), s.L * 0.5, s.L * (1 - 1e-15)]
    s.pos[2:40] = np.array([1.0, 1.0, 1.0]) * s.h * 0.25 + \
        np.random.default_rng(2).uniform(0, s.h * 3.5, (38, 3))
    prod.solver_initialize()
    maps = prod.type_maps()
    prod.solver_initialize_grid(s.n_grid, s.L, s.h, 1e-6, 1.0, 1.0, maps["method"]["LCG"], 0)
    prod.solver_initialize_particles(s.n_grid, 2, s.L, s.h, s.n_ions, 0, code, s.types, s.pos, s.vel,
                                     s.mass, s.charges, s.pot_params)
    prod.solver_initialize_integrator(s.n_ions, 1.0, 1200.0, 0.0, 1, 0)
    try:
        assert prod.solver_update_charges() == 0
        nbr = np.empty((s.n_ions, 64, 3), dtype=np.int64)
        prod.mzb_get_cic_neighbors(nbr)
        nbo = np.empty_like(nbr)
        oracle_lib.orc_spline_neighbors(s.pos, s.n_ions, s.n_grid, s.h, nbo)
        assert np.array_equal(nbr, nbo)
        q = np.empty((64, 64, 64))
        prod.get_q(q)
        qo = np.empty_like(q)
        oracle_lib.orc_spread_scheme(s.pos, s.charges, s.n_ions, 64, s.h, code, qo, None)
        if code == 1:
            assert np.array_equal(q, qo)
        else:
            assert rel(q, qo) < 1e-14
        phi = np.random.default_rng(3).standard_normal((64, 64, 64))
        prod.solver_set_field(phi)
        prod.solver_compute_forces_elec()
        fe = np.empty((s.n_ions, 3))
        prod.get_fcs_elec(fe)
        feo = np.empty_like(fe)
        oracle_lib.orc_force_scheme(phi, s.charges, s.pos, s.n_ions, 64, s.h, code, feo)
        if code == 1:
            assert np.array_equal(fe, feo)
        else:
            assert rel(fe, feo) < 1e-14
    finally:
        prod.solver_finalize()


@pytest.mark.parametrize("cas", ["SPL_QUADR", "SPL_CUBIC"])
def test_spline_crowded_tile(prod, oracle_lib, cas):
    """More than 1024 ions reach one 2 x 8 x 32 spreading tile (1100 ions packed around
    the box corner, wrapping across it): the tile kernel takes its slower path, which adds
    the ions in the same ascending order, so q stays bit-exact for the quadratic spline
    and within 1e-14 for the cubic one, and the field forces likewise."""
    code = {"SPL_QUADR": 1, "SPL_CUBIC": 2}[cas]
    s = make_system(10, 64, density=1.329, seed=37)
    rng = np.random.default_rng(5)
    box = np.array([1.5, 5.0, 20.0]) * s.h
    s.pos[:1100] = np.mod(rng.uniform(-box, box, (1100, 3)), s.L)
    s.pos[:1100] = np.where(s.pos[:1100] >= s.L, 0.0, s.pos[:1100])
    prod.solver_initialize()
    maps = prod.type_maps()
    prod.solver_initialize_grid(s.n_grid, s.L, s.h, 1e-6, 1.0, 1.0, maps["method"]["LCG"], 0)
    prod.solver_initialize_particles(s.n_grid, 2, s.L, s.h, s.n_ions, 0, code, s.types, s.pos, s.vel,
                                     s.mass, s.charges, s.pot_params)
    prod.solver_initialize_integrator(s.n_ions, 1.0, 1200.0, 0.0, 1, 0)
    try:
        assert prod.solver_update_charges() == 0
        q = np.empty((64, 64, 64))
        prod.get_q(q)
        qo = np.empty_like(q)
        oracle_lib.orc_spread_scheme(s.pos, s.charges, s.n_ions, 64, s.h, code, qo, None)
        if code == 1:
            assert np.array_equal(q, qo)
        else:
            assert rel(q, qo) < 1e-14
        phi = np.random.default_rng(6).standard_normal((64, 64, 64))
        prod.solver_set_field(phi)
        prod.solver_compute_forces_elec()
        fe = np.empty((s.n_ions, 3))
        prod.get_fcs_elec(fe)
        feo = np.empty_like(fe)
        oracle_lib.orc_force_scheme(phi, s.charges, s.pos, s.n_ions, 64, s.h, code, feo)
        if code == 1:
            assert np.array_equal(fe, feo)
        else:
            assert rel(fe, feo) < 1e-14
    finally:
        prod.solver_finalize()


@pytest.mark.parametrize("cas", ["SPL_QUADR", "SPL_CUBIC"])
def test_spline_md_250(prod, orc, cas):
    run_pair(prod, orc, make_system(5, 64, seed=13), 4, method="LCG", tol=1e-7, cas=cas)


@pytest.mark.parametrize("pot", ["LJ", "SC"])
def test_pair_potentials_250(prod, orc, pot):
    """Lennard-Jones and soft-core pair forces (forces.c:199-337) through MD steps."""
    run_pair(prod, orc, pair_system(5, 64, pot, seed=17), 4, method="LCG", tol=1e-7, pot=pot)


def test_maze_lcg_ssor_250(prod, orc):
    run_pair(prod, orc, make_system(5, 64, seed=3), 3, method="MAZE-LCG", precond="SSOR", tol=1e-9)


def test_maze_lcg_blockjacobi_250(prod, orc):
    """MAZE-LCG with the block-Jacobi preconditioner (grid 40^3, a multiple of the block)."""
    run_pair(prod, orc, make_system(5, 40, seed=4), 3, method="MAZE-LCG", precond="BLOCKJACOBI", tol=1e-9)
