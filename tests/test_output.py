"""Output and restart path (maze_poisson_b200/output.py) on the CPU oracle through the
reference's getters: the files carry the reference's columns
(maze_poisson/myio/output/csv.py:45-183), per-stride rows at the reference's instants
(base_out.py:136-152), and a run restarted from restart.csv / restart_field.csv
(solver.py:276-330, 371-409) continues like the uninterrupted run. pandas writes 16
significant digits, as it does for the reference, so values round-trip to ~5e-16."""
import os

import numpy as np
import pandas as pd
import pytest

from maze_poisson_b200.c_api import CAPI
from maze_poisson_b200.md import MDRun
from maze_poisson_b200.output import HEADERS, Outputs, read_restart, read_restart_field
from maze_poisson_b200.systems import make_system

# the reference's column lists, csv.py:47, 64, 76, 120, 134, 159, 179
REFERENCE_HEADERS = {
    "energy": "iter,K,V_notelec",
    "momentum": "iter,Px,Py,Pz",
    "temperature": "iter,T",
    "tot_force": "iter,Fx,Fy,Fz",
    "solute": "charge,iter,particle,x,y,z,vx,vy,vz,fx_elec,fy_elec,fz_elec",
    "restart": "type,x,y,z,vx,vy,vz",
    "restart_field": "phi_prev,phi",
}
TYPES = ["Na", "Cl"]


@pytest.fixture(scope="module")
def orc(oracle_path):
    return CAPI(oracle_path, extensions=False)


def run_with_outputs(capi, system, path, steps, stride, restart_step):
    run = MDRun(capi, system, method="LCG", tol=1e-9, integrator="VERLET")
    run.initialize()
    out = Outputs(capi, path, TYPES, system.n_grid, stride=stride, restart_step=restart_step).bind(system.n_ions)
    states = {}
    for i in range(steps):
        run.step()
        out.output(i, run.potential_notelec)
        states[i] = run.state()
    out.output(steps, run.potential_notelec, force=True)
    out.close()
    run.finalize()
    return states


def test_headers_rows_and_restart(orc, tmp_path):
    system = make_system(2, 16, seed=5)
    states = run_with_outputs(orc, system.copy(), str(tmp_path), steps=6, stride=2, restart_step=3)
    assert HEADERS.keys() == REFERENCE_HEADERS.keys()
    for name, header in REFERENCE_HEADERS.items():
        with open(os.path.join(tmp_path, f"{name}.csv")) as f:
            assert f.readline().strip() == header, name
    energy = pd.read_csv(tmp_path / "energy.csv")
    assert list(energy["iter"]) == [0, 2, 4, 6]  # every stride, and the final forced output
    assert np.isclose(energy["K"].iloc[1], states[2]["kinetic"], rtol=1e-15, atol=0)
    solute = pd.read_csv(tmp_path / "solute.csv")
    assert len(solute) == 4 * system.n_ions
    types, pos, vel = read_restart(tmp_path / "restart.csv", TYPES)
    assert np.array_equal(types, system.types)
    def close(a, b, tol=1e-15):
        return np.max(np.abs(a - b)) <= tol * np.max(np.abs(b))
    # velocities (~1e-4 a.u.) keep fewer significant digits in pandas' text than positions
    assert close(pos, states[3]["pos"]) and close(vel, states[3]["vel"], 1e-12)
    phi, phi_prev = read_restart_field(tmp_path / "restart_field.csv", system.n_grid)
    assert close(phi, states[3]["field"]) and close(phi_prev, states[3]["field_prev"])


def test_restart_continues_like_uninterrupted_run(orc, tmp_path):
    system = make_system(2, 16, seed=6)
    full = run_with_outputs(orc, system.copy(), str(tmp_path / "a"), steps=6, stride=10, restart_step=2)
    types, pos, vel = read_restart(tmp_path / "a" / "restart.csv", TYPES)
    phi, phi_prev = read_restart_field(tmp_path / "a" / "restart_field.csv", system.n_grid)
    restarted = system.copy()
    restarted.pos, restarted.vel = pos, vel
    run = MDRun(orc, restarted, method="LCG", tol=1e-9, integrator="VERLET")
    c = orc
    s = restarted
    maps = c.type_maps()
    c.solver_initialize()
    c.solver_initialize_grid(s.n_grid, s.L, s.h, run.tol, 1.0, 1.0, maps["method"]["LCG"], maps["precond"]["NONE"])
    c.solver_initialize_particles(s.n_grid, 2, s.L, s.h, s.n_ions, maps["potential"]["TF"], maps["cas"]["CIC"],
                                  s.types, s.pos, s.vel, s.mass, s.charges, s.pot_params)
    c.solver_initialize_integrator(s.n_ions, run.dt, run.T, run.gamma, maps["integrator"]["VERLET"], 0)
    c.solver_set_field(phi)
    c.solver_set_field_prev(phi_prev)
    run.update_charges()
    run.compute_forces()
    for _ in range(3):
        run.step()
    st = run.state()
    run.finalize()
    ref = full[5]
    for key in ("pos", "vel", "fcs_tot", "field"):
        err = np.max(np.abs(st[key] - ref[key])) / np.max(np.abs(ref[key]))
        assert err < 1e-12, (key, err)
