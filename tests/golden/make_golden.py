"""Generate the golden vectors that pin the oracle to the reference.

Runs in a container that has the reference tree: it drives the reference's own C
library (compiled from its sources by oracle/Makefile `ref`: -O2, no fast-math, no FMA)
single-threaded, through its exported functions and its facade, on seeded inputs, and
imports the reference's maze_poisson/linkedcell.py for the linked-cell layout. Small
arrays are stored whole; large fields as SHA-256 of their bytes plus samples.

    OMP_NUM_THREADS=1 python tests/golden/make_golden.py          # all fixtures
    OMP_NUM_THREADS=1 python tests/golden/make_golden.py --pb     # Poisson-Boltzmann ones
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
from maze_poisson_b200.systems import make_pb_system, make_system, pair_system, pb_settings  # noqa: E402
from oracle import loader  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))
REF_TREE = loader.REF_TREE  # MAZE_REFERENCE_ROOT, with the default in oracle/loader.py


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
    "maze_lcg_ssor": (2, 16, "MAZE-LCG", "SSOR", 1e-10, "VERLET", False, 3),
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


def ssor_kernel_cases(ref):
    """precond_ssor_apply (precond_ssor.c:1240-1252) on seeded inputs, n = 2..9, 16."""
    P = ctypes.c_void_p
    ref.precond_ssor_apply.argtypes = [P, P, ctypes.c_int, ctypes.c_int, ctypes.c_int]
    rng = np.random.default_rng(2024)
    out = {}
    for n in (2, 3, 4, 5, 6, 7, 8, 9, 16):
        x = rng.standard_normal((n, n, n))
        y = np.empty_like(x)
        ref.precond_ssor_apply(x.ctypes.data, y.ctypes.data, n, n, 0)
        out[f"n{n}_in"], out[f"n{n}_out"] = x, y
    return out


def pb_inputs(n, seed):
    """Seeded PB kernel inputs: face coefficients in [1, 78), screening in [0, 0.05), a
    field xt (tests/test_oracle_pin.py regenerates them the same way)."""
    rng = np.random.default_rng(seed)
    ex, ey, ez = (1.0 + 77.0 * rng.random((n, n, n)) for _ in range(3))
    k2 = 0.05 * rng.random((n, n, n))
    xt = rng.standard_normal((n, n, n))
    return ex, ey, ez, k2, xt


def pb_kernel_cases(ref):
    """The Poisson-Boltzmann grid kernels (laplace.c:77-145, plcg.c:169-238,
    multigrid_pb.c) on seeded positive face coefficients and screening terms."""
    P = ctypes.c_void_p
    D, I = ctypes.c_double, ctypes.c_int
    ref.laplace_filter_pb.argtypes = [P, P, I, I, P, P, P, P]
    ref.smooth_pb_rbgs.argtypes = [P, P, I, I, D, P, P, P, P]
    ref.restriction_eps.argtypes = [P, P, I, I, I]
    ref.restriction_k2screen.argtypes = [P, P, I, I, I]
    ref.conj_grad_pb.argtypes = [P, P, P, D, I, I, P, P, P, P]
    ref.conj_grad_pb.restype = I
    ref.multigrid_pb_apply.argtypes = [P, P, I, I, I, I, P, P, P, P]
    ref.solver_initialize_grid.argtypes = [I, D, D, D, D, D, I, I]
    out = {}
    for n, seed in ((16, 4321), (32, 4322)):
        ref.solver_initialize()
        ref.solver_initialize_grid(n, 1.0, 1.0 / n, 1e-7, 1.0, 1.0, 2 if n == 32 else 0, 0)
        ex, ey, ez, k2, xt = pb_inputs(n, seed)
        keep = [halo(a) for a in (ex, ey, ez)]
        cp = [k[1] for k in keep] + [k2.ctypes.data]
        xtb, xtp = halo(xt)
        b = np.zeros((n, n, n))
        ref.laplace_filter_pb(xtp, b.ctypes.data, n, n, *cp)
        out[f"n{n}_seed"] = np.array(seed)
        if n == 16:
            out["n16_b"] = b.copy()
            rng = np.random.default_rng(99)
            rhs = rng.standard_normal((n, n, n))
            x0 = rng.standard_normal((n, n, n))
            xb, xp = halo(x0)
            ref.smooth_pb_rbgs(rhs.ctypes.data, xp, n, n, 3.0, *cp)
            out["rbgs_out"] = xb[1:-1].copy()
            for axis, (name, arr) in enumerate((("ex", ex), ("ey", ey), ("ez", ez))):
                ab, ap = halo(arr)
                c = np.zeros((n // 2,) * 3)
                ref.restriction_eps(ap, c.ctypes.data, n, n, axis)
                out[f"restrict_{name}"] = c
            c = np.zeros((n // 2,) * 3)
            ref.restriction_k2screen(k2.ctypes.data, c.ctypes.data, n, n, 0)
            out["restrict_k2"] = c
            zb, zp = halo(np.zeros((n, n, n)))
            x = np.zeros((n, n, n))
            it = ref.conj_grad_pb(b.ctypes.data, zp, x.ctypes.data, 1e-9, n, n, *cp)
            out["cg_x"], out["cg_iters"] = x, np.array(it)
        else:
            out["n32_b_sha"] = np.array(sha(b))
            xb, xp = halo(np.zeros((n, n, n)))
            ref.multigrid_pb_apply(b.ctypes.data, xp, n, n, 0, 4, *cp)
            out["mg_x_sha"] = np.array(sha(xb[1:-1]))
            out["mg_x_sample"] = xb[1:-1].reshape(-1)[::997].copy()
        ref.solver_finalize()
        del keep
    return out


PB_SCENARIOS = {
    # name: (n_ions, n_grid, box [A], seed, method, tol, steps, nonpolar, eps_s)
    "pb_lcg": (8, 32, 16.0, 3, "LCG", 1e-10, 2, 1, 78.4),
    "pb_maze_lcg": (8, 32, 16.0, 3, "MAZE-LCG", 1e-10, 2, 0, 78.4),
    "pb_multigrid": (8, 32, 16.0, 3, "MULTIGRID", 1e-8, 2, 1, 78.4),
    "pb_maze_multigrid": (8, 32, 16.0, 3, "MAZE-MULTIGRID", 1e-8, 2, 1, 78.4),
}


def pb_run(capi, spec):
    """The MD run of a PB scenario (implicit solvent, Tosi-Fumi pairs, Verlet at 300 K)."""
    n_ions, ng, box, seed, method, tol, steps, nonpolar, eps_s = spec
    system = make_pb_system(n_ions, ng, box, T=300.0, seed=seed)
    return MDRun(capi, system, method=method, tol=tol, integrator="VERLET", T=300.0, eps_s=eps_s,
                 eps_int=1.0, pb=pb_settings(system, eps_s=eps_s, nonpolar=nonpolar))


def pb_scenario(ref_path, spec):
    run = pb_run(CAPI(ref_path, extensions=False), spec)
    run.initialize()
    rec = {}
    for s in range(-1, spec[6]):
        if s >= 0:
            run.step()
        st = run.state()
        tag = "init" if s < 0 else f"s{s}"
        for key in ("pos", "vel", "fcs_tot", "fcs_elec", "fcs_noel", "fcs_db", "fcs_ib", "fcs_np"):
            rec[f"{tag}_{key}"] = st[key]
        rec[f"{tag}_iters"] = np.array(-2 if st["n_iters"] is None else st["n_iters"])
        rec[f"{tag}_field_sha"] = np.array(sha(st["field"]))
        rec[f"{tag}_field_sample"] = st["field"].reshape(-1)[::101].copy()
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
    if "--pb" in sys.argv:
        loader.build(ref=True)
        ref = ctypes.CDLL(loader.REF_SO, mode=ctypes.RTLD_LOCAL)
        np.savez_compressed(os.path.join(OUT, "pb_kernels.npz"), **pb_kernel_cases(ref))
        for name, spec in PB_SCENARIOS.items():
            np.savez_compressed(os.path.join(OUT, f"md_{name}.npz"), **pb_scenario(loader.REF_SO, spec))
            print(name, "done", flush=True)
        with open(os.path.join(OUT, "pb_scenarios.json"), "w") as f:
            json.dump({k: list(v) for k, v in PB_SCENARIOS.items()}, f, indent=1)
        return
    only = None
    if "--only" in sys.argv:  # regenerate just these scenarios (comma-separated)
        only = set(sys.argv[sys.argv.index("--only") + 1].split(","))
    loader.build(ref=True)
    if only is None:
        ref = ctypes.CDLL(loader.REF_SO, mode=ctypes.RTLD_LOCAL)
        data = kernel_cases(ref)
        np.savez_compressed(os.path.join(OUT, "kernels.npz"), **data)
    if only is None or "ssor_kernels" in only:
        ref = ctypes.CDLL(loader.REF_SO, mode=ctypes.RTLD_LOCAL)
        np.savez_compressed(os.path.join(OUT, "ssor_kernels.npz"), **ssor_kernel_cases(ref))
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
