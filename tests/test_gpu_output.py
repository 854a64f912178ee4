"""Asynchronous output snapshots (mzb_snapshot_begin / _fetch): a snapshot holds exactly
the values the blocking getters return at the instant it was queued, even after further
MD steps overwrite the device arrays; the reference-format files written from snapshots
equal the files written from the getters byte for byte."""
import filecmp

import numpy as np
import pytest

from maze_poisson_b200.c_api import CAPI
from maze_poisson_b200.md import MDRun
from maze_poisson_b200.output import Outputs
from maze_poisson_b200.systems import make_system

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def prod(product_path):
    return CAPI(product_path)


def test_snapshot_equals_getters(prod):
    system = make_system(5, 64, seed=9)
    h = prod.mzb_system_create()
    run = MDRun(prod, system, method="LCG", tol=1e-10, integrator="OVRVO", thermostat=True, precision=1)
    run.initialize()
    try:
        for _ in range(3):
            run.step()
        slot = prod.mzb_snapshot_begin(31)
        assert slot in (0, 1)
        ref = run.state()
        mom = np.empty(3)
        prod.get_momentum(mom)
        K, T, V = prod.get_kinetic_energy(), prod.get_temperature(), run.potential_notelec
        for _ in range(3):  # the device arrays move on; the snapshot must not
            run.step()
        n, g = system.n_ions, system.n_grid
        out = {k: np.empty((n, 3)) for k in ("pos", "vel", "fcs_elec", "fcs_noel", "fcs_tot")}
        sc = np.empty(8)
        phi, phi_prev = np.empty((g, g, g)), np.empty((g, g, g))
        got = prod.mzb_snapshot_fetch(slot, *(out[k].ctypes.data for k in ("pos", "vel", "fcs_elec", "fcs_noel",
                                                                        "fcs_tot")),
                                      sc.ctypes.data, phi.ctypes.data, phi_prev.ctypes.data)
        assert got == 31
        for k, a in out.items():
            assert np.array_equal(a, ref[k]), k
        assert np.array_equal(phi, ref["field"]) and np.array_equal(phi_prev, ref["field_prev"])
        assert sc[1] == V and sc[2] == K and sc[6] == T and np.array_equal(sc[3:6], mom)
        assert prod.mzb_snapshot_fetch(slot, *([None] * 8)) == -1
    finally:
        prod.mzb_system_destroy(h)


def test_files_from_snapshots_equal_files_from_getters(prod, tmp_path):
    paths = []
    for mode in (True, False):
        system = make_system(4, 64, seed=12)
        h = prod.mzb_system_create()
        run = MDRun(prod, system, method="LCG", tol=1e-10, integrator="VERLET", precision=1)
        run.initialize()
        path = tmp_path / ("async" if mode else "sync")
        out = Outputs(prod, str(path), ["Na", "Cl"], system.n_grid, stride=2, restart_step=5,
                      use_snapshots=mode).bind(system.n_ions)
        for i in range(8):
            run.step()
            out.output(i, run.potential_notelec)
        out.output(8, run.potential_notelec, force=True)
        out.close()
        prod.mzb_system_destroy(h)
        paths.append(path)
    for name in ("energy", "momentum", "temperature", "tot_force", "solute", "restart", "restart_field"):
        assert filecmp.cmp(paths[0] / f"{name}.csv", paths[1] / f"{name}.csv", shallow=False), name
