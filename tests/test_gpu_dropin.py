"""Drop-in check through the reference's own Python: its SolverMD (maze_poisson/solver.py
with its ctypes bindings, maze_poisson/c_api) loads `maze_poisson/libmaze_poisson.so`
(c_api/__init__.py:44-46). A copy of the reference's package, staged unchanged by
`make -C oracle ref` into oracle/_ref/py, gets this build's library at that path and runs
its own initialize() and md_loop_iter(); a second copy gets the CPU oracle's library
instead. Both runs read the same input files (written as the reference expects them:
species.csv, tosi_fumi.csv, positions and velocities in a CSV) and must agree within
1e-10 after every step. Skipped where the staged package is absent."""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

from conftest import ROOT
from maze_poisson_b200.systems import make_system, write_reference_inputs

pytestmark = pytest.mark.gpu
REF_PKG = os.path.join(ROOT, "oracle", "_ref", "py", "maze_poisson")

DRIVER = r"""
import json, os, sys
import numpy as np
sys.path.insert(0, {pkg_parent!r})
os.chdir({work!r})
from maze_poisson.myio.input.dct import initialize_from_dict
from maze_poisson.solver import SolverMD
from maze_poisson.c_api import capi
gset, outset, mdv = initialize_from_dict({settings!r})
solver = SolverMD(gset, mdv, outset)
solver.initialize()
out = {{}}
def grab(tag):
    for name in ("pos", "vel", "fcs_tot", "fcs_elec"):
        a = np.empty(({n_p}, 3))
        getattr(capi, "get_" + name)(a)
        out[tag + name] = a
    phi = np.empty(({n}, {n}, {n}))
    capi.get_field(phi)
    out[tag + "field"] = phi
    out[tag + "kinetic"] = np.array(capi.get_kinetic_energy())
grab("init_")
iters = []
for s in range({steps}):
    solver.md_loop_iter()
    iters.append(solver.n_iters)
    grab(f"s{{s}}_")
out["iters"] = np.array(iters)
np.savez({out!r}, **out)
print(json.dumps({{"library": capi.path, "iters": iters}}))
"""


def run_reference_solvermd(tmp, tag, library, system, settings, steps):
    import shutil
    parent = os.path.join(tmp, tag)
    shutil.copytree(REF_PKG, os.path.join(parent, "maze_poisson"))
    os.symlink(library, os.path.join(parent, "maze_poisson", "libmaze_poisson.so"))
    work = os.path.join(tmp, tag + "_work")
    os.makedirs(work)
    out = os.path.join(tmp, tag + ".npz")
    code = DRIVER.format(pkg_parent=parent, work=work, settings=settings, n_p=system.n_ions, n=system.n_grid,
                         steps=steps, out=out)
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=900,
                       env=dict(os.environ, MZB_QUIET="1"))
    assert r.returncode == 0, r.stderr[-3000:]
    info = json.loads(r.stdout.strip().splitlines()[-1])
    assert os.path.realpath(info["library"]) == os.path.realpath(library)
    return dict(np.load(out))


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


@pytest.mark.skipif(not os.path.isdir(REF_PKG), reason="the reference's Python package is not staged")
@pytest.mark.parametrize("method,integrator", [("LCG", "VERLET"), ("MAZE-MULTIGRID", "VERLET")])
def test_reference_solvermd_drives_this_library(tmp_path, product_path, oracle_path, method, integrator):
    system = make_system(5, 64, seed=3)
    inputs = os.path.join(str(tmp_path), "inputs")
    write_reference_inputs(system, inputs)
    settings = {
        "grid_setting": {"N": system.n_grid, "N_p": system.n_ions, "N_typs": 2, "L": system.L,
                         "input_file": os.path.join(inputs, "input.csv"),
                         "particles_file": os.path.join(inputs, "species.csv"), "cas": "CIC"},
        "md_variables": {"N_steps": 4, "T": 1200.0, "dt_fs": 1.0, "tol": 1e-9, "method": method,
                         "integrator": integrator, "potential": "TF",
                         "potential_params_file": os.path.join(inputs, "tosi_fumi.csv"), "thermostat": False},
        "output_settings": {"path": os.path.join(str(tmp_path), "out") + "/", "stride": 1000},
    }
    steps = 4
    a = run_reference_solvermd(str(tmp_path), "product", product_path, system, settings, steps)
    b = run_reference_solvermd(str(tmp_path), "oracle", oracle_path, system, settings, steps)
    assert np.all(np.abs(a["iters"] - b["iters"]) <= 1), (a["iters"], b["iters"])
    for tag in ["init_"] + [f"s{s}_" for s in range(steps)]:
        for key in ("pos", "vel", "fcs_tot", "fcs_elec", "field"):
            assert rel(a[tag + key], b[tag + key]) < 1e-10, (tag, key, rel(a[tag + key], b[tag + key]))
        assert abs(a[tag + "kinetic"] - b[tag + "kinetic"]) <= 1e-10 * abs(b[tag + "kinetic"])
