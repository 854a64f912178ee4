"""Generate the golden vectors that pin the oracle to the reference.

Runs in a container that has the reference tree: it drives the reference's own C
library (compiled from its sources by oracle/Makefile `ref`: -O2, no fast-math, no FMA)
single-threaded, through its exported functions and its facade, on seeded inputs, and
imports the reference's maze_poisson/linkedcell.py for the linked-cell layout. Small
arrays are stored whole; large fields as SHA-256 of their bytes plus samples.

    OMP_NUM_THREADS=1 python tests/golden/make_golden.py
"""
import ctypes
import hashlib
import importlib.util
import json
import os
import sys

os.environ["OMP_NUM_THREADS"] = "1"

import numpy as np  # noqa: E402

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from maze_poisson_b200.c_api import CAPI  # noqa: E402
from maze_poisson_b200.md import MDRun  # noqa: E402
from maze_poisson_b200.systems import make_system, pair_system  # noqa: E402
from oracle import loader  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))
REF_TREE = "/root/reference"


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def halo(a):
    """Copy an n^3 array into an (n+2, n, n) buffer; return (buffer, interior pointer)."""
    n = a.shape[0]
    buf = np.zeros((n + 2, n, n))
    buf[1:-1] = a
    ptr = buf.ctypes.data + n * n * 8
    return buf, ptr


def kernel_cases(ref):
    P = ctypes.c_void_p
    D, I = ctypes.c_double, ctypes.c_int
    ref.laplace_filter.argtypes = [P, P, I, I]
    ref.smooth_rbgs.argtypes = [P, P, I, I, D]
    ref.restriction_27pt.argtypes = [P, P, I, I, I]
    ref.prolong_trilinear.argtypes = [P, P, I, I, I, I, I]
    ref.conj_grad.argtypes = [P, P, P, D, I, I]
    ref.conj_grad.restype = I
    ref.multigrid_apply.argtypes = [P, P, I, I, I, I]
    ref.solver_initialize_grid.argtypes = [I, D, D, D, D, D, I, I]
    # the kernels read get_n_start() from a grid: initialise one (serial: n_start = 0)
    ref.solver_initialize()
    out = {}
    rng = np.random.default_rng(1234)

    n = 16
    u = rng.standard_normal((n, n, n))
    ub, up = halo(u)
    o = np.zeros((n, n, n))
    ref.solver_initialize_grid(n, 1.0, 1.0 / n, 1e-7, 1.0, 1.0, 0, 0)
    ref.laplace_filter(up, o.ctypes.data, n, n)
    out["laplace_in"], out["laplace_out"] = u, o.copy()

    rhs = rng.standard_normal((n, n, n))
    x0 = rng.standard_normal((n, n, n))
    xb, xp = halo(x0)
    rb, rp = halo(rhs)
    ref.smooth_rbgs(rp, xp, n, n, 3.0)
    out["rbgs_rhs"], out["rbgs_x0"], out["rbgs_out"] = rhs, x0, xb[1:-1].copy()

    f = rng.standard_normal((n, n, n))
    fb, fp = halo(f)
    c = np.zeros((n // 2,) * 3)
    ref.restriction_27pt(fp, c.ctypes.data, n, n, 0)
    out["restrict_in"], out["restrict_out"] = f, c

    nc = 8
    cin = rng.standard_normal((nc, nc, nc))
    cb, cp = halo(cin)
    fo = np.zeros((2 * nc,) * 3)
    ref.prolong_trilinear(cp, fo.ctypes.data, nc, nc, 2 * nc, 2 * nc, 0)
    out["prolong_in"], out["prolong_out"] = cin, fo

    xt = rng.standard_normal((n, n, n))
    xtb, xtp = halo(xt)
    b = np.zeros((n, n, n))
    ref.laplace_filter(xtp, b.ctypes.data, n, n)
    z = np.zeros((n, n, n))
    zb, zp = halo(z)
    x = np.zeros((n, n, n))
    it = ref.conj_grad(b.ctypes.data, zp, x.ctypes.data, 1e-9, n, n)
    out["cg_b"], out["cg_x"], out["cg_iters"] = b, x, np.array(it)
    ref.solver_finalize()

    # one V-cycle needs n/2 >= 16
    n = 32
    ref.solver_initialize()
    ref.solver_initialize_grid(n, 1.0, 1.0 / n, 1e-7, 1.0, 1.0, 2, 0)
    xt = rng.standard_normal((n, n, n))
    xtb, xtp = halo(xt)
    b = np.zeros((n, n, n))
    ref.laplace_filter(xtp, b.ctypes.data, n, n)
    xb, xp = halo(np.zeros((n, n, n)))
    ref.multigrid_apply(b.ctypes.data, xp, n, n, 0, 3)
    out["mg_seed_x"], out["mg_x_sha"] = xt, np.array(sha(xb[1:-1]))
    out["mg_x_sample"] = xb[1:-1].reshape(-1)[::997].copy()
    ref.solver_finalize()
    return out


SCENARIOS = {
    # name: (ncell, n_grid, method, precond, tol, integrator, thermostat, steps)
    "lcg_verlet": (2, 16, "LCG", "NONE", 1e-10, "VERLET", False, 5),
    "maze_lcg": (2, 16, "MAZE-LCG", "NONE", 1e-10, "VERLET", False, 5),
    "maze_lcg_jacobi": (2, 16, "MAZE-LCG", "JACOBI", 1e-10, "VERLET", False, 3),
    "maze_lcg_mg": (2, 32, "MAZE-LCG", "MG", 1e-9, "VERLET", False, 2),
    "multigrid": (2, 32, "MULTIGRID", "NONE", 1e-8, "VERLET", False, 3),
    "maze_multigrid": (2, 32, "MAZE-MULTIGRID", "NONE", 1e-8, "VERLET", False, 3),
    "ovrvo_nothermo": (2, 16, "LCG", "NONE", 1e-10, "OVRVO", False, 5),
    "verlet_thermo": (2, 16, "LCG", "NONE", 1e-10, "VERLET", True, 3),
    # B-spline charge assignment (charges.c:16-38, particles.c:348-385)
    "spl_quadr": (2, 16, "LCG", "NONE", 1e-10, "VERLET", False, 3, "SPL_QUADR"),
    "spl_cubic": (2, 16, "LCG", "NONE", 1e-10, "VERLET", False, 3, "SPL_CUBIC"),
    # Lennard-Jones (parameters laid out so that the reference's stride-4 read sees the
    # same table as the stride-2 layout, systems.lj_params_au) and soft-core pair
    # potentials (forces.c:199-337)
    "lj_fluid": (2, 16, "LCG", "NONE", 1e-10, "VERLET", False, 4, "CIC", "LJ"),
    "sc_melt": (2, 16, "LCG", "NONE", 1e-10, "VERLET", False, 4, "CIC", "SC"),
}


def scenario(ref_path, name, spec):
    ncell, ng, method, precond, tol, itg, thermo, steps = spec[:8]
    cas = spec[8] if len(spec) > 8 else "CIC"
    pot = spec[9] if len(spec) > 9 else "TF"
    system = pair_system(ncell, ng, pot, density=1.379, T=1200.0, seed=7)
    run = MDRun(CAPI(ref_path, extensions=False), system, method=method, precond=precond, tol=tol,
                integrator=itg, thermostat=thermo, cas=cas, pot=pot)
    run.initialize()
    st = run.state()
    rec = {"init_q_sha": np.array(sha(st["q"])), "init_field_sha": np.array(sha(st["field"])),
           "init_fcs_tot": st["fcs_tot"], "init_fcs_elec": st["fcs_elec"],
           "init_fcs_noel": st["fcs_noel"], "init_pos": st["pos"], "init_vel": st["vel"],
           "init_potential": np.array(st["potential_notelec"])}
    if ng == 16:
        rec["init_q"], rec["init_field"] = st["q"], st["field"]
    for s in range(steps):
        run.step()
        st = run.state()
        rec[f"s{s}_pos"], rec[f"s{s}_vel"] = st["pos"], st["vel"]
        rec[f"s{s}_fcs_tot"], rec[f"s{s}_iters"] = st["fcs_tot"], np.array(st["n_iters"])
        rec[f"s{s}_potential"], rec[f"s{s}_kinetic"] = (np.array(st["potential_notelec"]),
                                                        np.array(st["kinetic"]))
        rec[f"s{s}_field_sha"] = np.array(sha(st["field"]))
        rec[f"s{s}_field_sample"] = st["field"].reshape(-1)[::101].copy()
    run.finalize()
    return rec


def linked_cells():
    spec = importlib.util.spec_from_file_location(
        "ref_linkedcell", os.path.join(REF_TREE, "maze_poisson", "linkedcell.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    system = make_system(5, 64, density=1.379, seed=11)

    class _P:
        def __init__(self, p):
            self.pos = p
    out = {}
    for nc in (3, 4):
        lc = mod.LinkedCell(system.L / nc * 0.9999999, system.L, system.n_ions)
        assert lc.side_cell_num == nc
        lc.update_lists([_P(p) for p in system.pos])
        out[f"lc{nc}_header"] = lc.header.astype(np.int64)
        out[f"lc{nc}_link"] = lc.link.astype(np.int64)
    out["lc_pos"], out["lc_L"] = system.pos, np.array(system.L)
    return out


def main():
    only = None
    if "--only" in sys.argv:  # regenerate just these scenarios (comma-separated)
        only = set(sys.argv[sys.argv.index("--only") + 1].split(","))
    loader.build(ref=True)
    if only is None:
        ref = ctypes.CDLL(loader.REF_SO, mode=ctypes.RTLD_LOCAL)
        data = kernel_cases(ref)
        np.savez_compressed(os.path.join(OUT, "kernels.npz"), **data)
    for name, spec in SCENARIOS.items():
        if only is not None and name not in only:
            continue
        rec = scenario(loader.REF_SO, name, spec)
        np.savez_compressed(os.path.join(OUT, f"md_{name}.npz"), **rec)
        print(name, "done", flush=True)
    if only is None:
        np.savez_compressed(os.path.join(OUT, "linked_cells.npz"), **linked_cells())
    with open(os.path.join(OUT, "scenarios.json"), "w") as f:
        json.dump({k: list(v) for k, v in SCENARIOS.items()}, f, indent=1)


if __name__ == "__main__":
    main()
