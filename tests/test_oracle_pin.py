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
from maze_poisson_b200.systems import make_system, pair_system


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
