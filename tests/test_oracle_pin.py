"""Pin the CPU oracle to the reference: every golden vector under tests/golden was made by
the reference's own C (tests/golden/make_golden.py); the oracle must reproduce each one
bit for bit (same operation order, no FMA, serial reductions)."""
import hashlib
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN
from maze_poisson_b200.c_api import CAPI
from maze_poisson_b200.md import MDRun
from maze_poisson_b200.systems import make_pb_system, make_system, pair_system, pb_settings


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


@pytest.fixture(scope="module")
def K():
    return np.load(os.path.join(GOLDEN, "kernels.npz"))


def test_laplace_bitexact(oracle_lib, K):
    u = np.ascontiguousarray(K["laplace_in"])
    out = np.empty_like(u)
    oracle_lib.orc_laplace(u, out, 16)
    assert np.array_equal(out, K["laplace_out"])


def test_rbgs_bitexact(oracle_lib, K):
    x = np.ascontiguousarray(K["rbgs_x0"]).copy()
    oracle_lib.orc_smooth_rbgs(np.ascontiguousarray(K["rbgs_rhs"]), x, 16, 3)
    assert np.array_equal(x, K["rbgs_out"])


def test_restriction_bitexact(oracle_lib, K):
    out = np.empty((8, 8, 8))
    oracle_lib.orc_restrict27(np.ascontiguousarray(K["restrict_in"]), out, 16)
    assert np.array_equal(out, K["restrict_out"])


def test_prolong_bitexact(oracle_lib, K):
    out = np.empty((16, 16, 16))
    oracle_lib.orc_prolong_trilinear(np.ascontiguousarray(K["prolong_in"]), out, 8)
    assert np.array_equal(out, K["prolong_out"])


def test_conj_grad_bitexact(oracle_lib, K):
    b = np.ascontiguousarray(K["cg_b"])
    x = np.empty_like(b)
    it = oracle_lib.orc_conj_grad(b, np.zeros_like(b), x, 1e-9, 16)
    assert it == int(K["cg_iters"])
    assert np.array_equal(x, K["cg_x"])


def test_vcycle_bitexact(oracle_lib, K):
    xt = np.ascontiguousarray(K["mg_seed_x"])
    b = np.empty_like(xt)
    oracle_lib.orc_laplace(xt, b, 32)
    x = np.zeros_like(xt)
    oracle_lib.orc_mg_apply(b, x, 32, 3)
    assert np.array_equal(x.reshape(-1)[::997], K["mg_x_sample"])
    assert sha(x) == str(K["mg_x_sha"])


def test_ssor_bitexact(oracle_lib):
    g = np.load(os.path.join(GOLDEN, "ssor_kernels.npz"))
    for n in (2, 3, 4, 5, 6, 7, 8, 9, 16):
        x = np.ascontiguousarray(g[f"n{n}_in"])
        y = np.empty_like(x)
        oracle_lib.orc_ssor_apply(x, y, n)
        assert np.array_equal(y, g[f"n{n}_out"]), n


SCEN = json.load(open(os.path.join(GOLDEN, "scenarios.json")))


@pytest.mark.parametrize("name", sorted(SCEN))
def test_md_scenario_bitexact(oracle_path, name):
    ncell, ng, method, precond, tol, itg, thermo, steps = SCEN[name][:8]
    cas = SCEN[name][8] if len(SCEN[name]) > 8 else "CIC"
    pot = SCEN[name][9] if len(SCEN[name]) > 9 else "TF"
    g = np.load(os.path.join(GOLDEN, f"md_{name}.npz"))
    system = pair_system(ncell, ng, pot, density=1.379, T=1200.0, seed=7)
    run = MDRun(CAPI(oracle_path, extensions=False), system, method=method, precond=precond, tol=tol,
                integrator=itg, thermostat=thermo, cas=cas, pot=pot)
    run.initialize()
    try:
        st = run.state()
        assert sha(st["q"]) == str(g["init_q_sha"])
        assert sha(st["field"]) == str(g["init_field_sha"])
        for key in ("fcs_tot", "fcs_elec", "fcs_noel", "pos", "vel"):
            assert np.array_equal(st[key], g["init_" + key]), key
        assert st["potential_notelec"] == float(g["init_potential"])
        for s in range(steps):
            run.step()
            st = run.state()
            assert st["n_iters"] == int(g[f"s{s}_iters"]), s
            for key in ("pos", "vel", "fcs_tot"):
                assert np.array_equal(st[key], g[f"s{s}_{key}"]), (s, key)
            assert st["potential_notelec"] == float(g[f"s{s}_potential"])
            assert st["kinetic"] == float(g[f"s{s}_kinetic"])
            assert sha(st["field"]) == str(g[f"s{s}_field_sha"]), s
    finally:
        run.finalize()


def test_linked_cells_match_reference_chain(oracle_lib):
    """The oracle's CSR cells list each cell's ions ascending; the reference's header/link
    chain (maze_poisson/linkedcell.py) lists them descending from the header."""
    g = np.load(os.path.join(GOLDEN, "linked_cells.npz"))
    pos = np.ascontiguousarray(g["lc_pos"])
    L = float(g["lc_L"])
    for nc in (3, 4):
        start = np.empty(nc ** 3 + 1, dtype=np.int32)
        ions = np.empty(len(pos), dtype=np.int32)
        oracle_lib.orc_cell_list(pos, len(pos), L, nc, start, ions)
        header = g[f"lc{nc}_header"].reshape(-1)
        link = g[f"lc{nc}_link"]
        for c in range(nc ** 3):
            chain = []
            p = header[c]
            while p >= 0:
                chain.append(int(p))
                p = link[p]
            assert list(ions[start[c]:start[c + 1]]) == chain[::-1]


# ---------------------------------------------------------------- Poisson-Boltzmann
def pb_inputs(n, seed):
    """The seeded inputs make_golden.py gave the reference's PB kernels."""
    rng = np.random.default_rng(seed)
    ex, ey, ez = (1.0 + 77.0 * rng.random((n, n, n)) for _ in range(3))
    k2 = 0.05 * rng.random((n, n, n))
    xt = rng.standard_normal((n, n, n))
    return ex, ey, ez, k2, xt


@pytest.fixture(scope="module")
def PBK():
    return np.load(os.path.join(GOLDEN, "pb_kernels.npz"))


def test_pb_grid_kernels_bitexact(oracle_lib, PBK):
    n = 16
    ex, ey, ez, k2, xt = pb_inputs(n, int(PBK["n16_seed"]))
    b = np.empty_like(xt)
    oracle_lib.orc_laplace_pb(xt, b, ex, ey, ez, k2, n)
    assert np.array_equal(b, PBK["n16_b"])
    rng = np.random.default_rng(99)
    rhs = rng.standard_normal((n, n, n))
    x = rng.standard_normal((n, n, n))
    oracle_lib.orc_smooth_pb(rhs, x, n, 3, ex, ey, ez, k2)
    assert np.array_equal(x, PBK["rbgs_out"])
    for axis, (name, arr) in enumerate((("ex", ex), ("ey", ey), ("ez", ez))):
        c = np.empty((8, 8, 8))
        oracle_lib.orc_restrict_eps(arr, c, n, axis)
        assert np.array_equal(c, PBK[f"restrict_{name}"]), name
    c = np.empty((8, 8, 8))
    oracle_lib.orc_restrict_k2(k2, c, n)
    assert np.array_equal(c, PBK["restrict_k2"])
    x = np.empty_like(b)
    it = oracle_lib.orc_conj_grad_pb(b, np.zeros_like(b), x, 1e-9, n, ex, ey, ez, k2)
    assert it == int(PBK["cg_iters"])
    assert np.array_equal(x, PBK["cg_x"])


def test_pb_vcycle_bitexact(oracle_lib, PBK):
    n = 32
    ex, ey, ez, k2, xt = pb_inputs(n, int(PBK["n32_seed"]))
    b = np.empty_like(xt)
    oracle_lib.orc_laplace_pb(xt, b, ex, ey, ez, k2, n)
    assert sha(b) == str(PBK["n32_b_sha"])
    x = np.zeros_like(xt)
    oracle_lib.orc_mg_pb_apply(b, x, n, 4, ex, ey, ez, k2)
    assert np.array_equal(x.reshape(-1)[::997], PBK["mg_x_sample"])
    assert sha(x) == str(PBK["mg_x_sha"])


PB_SCEN = json.load(open(os.path.join(GOLDEN, "pb_scenarios.json")))


def pb_run(capi, spec):
    """The MD run of a PB scenario, built as make_golden.py builds it."""
    n_ions, ng, box, seed, method, tol, steps, nonpolar, eps_s = spec
    system = make_pb_system(n_ions, ng, box, T=300.0, seed=seed)
    return MDRun(capi, system, method=method, tol=tol, integrator="VERLET", T=300.0, eps_s=eps_s,
                 eps_int=1.0, pb=pb_settings(system, eps_s=eps_s, nonpolar=nonpolar))


@pytest.mark.parametrize("name", sorted(PB_SCEN))
def test_pb_md_scenario_bitexact(oracle_path, name):
    spec = PB_SCEN[name]
    g = np.load(os.path.join(GOLDEN, f"md_{name}.npz"))
    run = pb_run(CAPI(oracle_path, extensions=False), spec)
    run.initialize()
    try:
        for s in range(-1, spec[6]):
            if s >= 0:
                run.step()
            st = run.state()
            tag = "init" if s < 0 else f"s{s}"
            iters = -2 if st["n_iters"] is None else st["n_iters"]
            assert iters == int(g[f"{tag}_iters"]), tag
            for key in ("pos", "vel", "fcs_tot", "fcs_elec", "fcs_noel", "fcs_db", "fcs_ib", "fcs_np"):
                assert np.array_equal(st[key], g[f"{tag}_{key}"]), (tag, key)
            assert sha(st["field"]) == str(g[f"{tag}_field_sha"]), tag
    finally:
        run.finalize()


def test_blockjacobi_inverse_matches_lapack(oracle_lib):
    """Block-Jacobi parity is unpinned: the reference inverts its block with LAPACK's
    dgetri, which this image lacks, so its block-Jacobi path cannot run here. The oracle's
    Gauss-Jordan inverse is checked against LAPACK's (numpy) instead, and its product
    against a numpy restatement of the reorder + dgemm (precond_blockjacobi.c:79-206)."""
    B = 10
    A = np.zeros((1000, 1000))
    for i in range(B):
        for j in range(B):
            for k in range(B):
                r = (i * B + j) * B + k
                A[r, r] = -6.0
                for di, dj, dk in ((1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1)):
                    ii, jj, kk = i + di, j + dj, k + dk
                    if 0 <= ii < B and 0 <= jj < B and 0 <= kk < B:
                        A[r, (ii * B + jj) * B + kk] = 1.0
    inv = np.empty((1000, 1000))
    oracle_lib.orc_blockjacobi_inverse(inv)
    ref = np.linalg.inv(A)
    assert np.max(np.abs(inv - ref)) <= 1e-14 * np.max(np.abs(ref))
    n = 20
    x = np.random.default_rng(1).standard_normal((n, n, n))
    y = np.empty_like(x)
    oracle_lib.orc_blockjacobi_apply(x, y, n)
    blocks = x.reshape(2, 10, 2, 10, 2, 10).transpose(0, 2, 4, 1, 3, 5).reshape(8, 1000)
    yy = (blocks @ ref).reshape(2, 2, 2, 10, 10, 10).transpose(0, 3, 1, 4, 2, 5).reshape(n, n, n)
    assert np.max(np.abs(y - yy)) <= 1e-13 * np.max(np.abs(yy))
