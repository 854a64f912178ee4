"""Several resident systems and the batched step.

The same systems are stepped alone (each through the per-call reference path with the
FP32+refine field solve) and together in mzb_batch_step (CUDA graph per step, one
cooperative launch for all field solves), after mzb_batch_autotune has picked the team
partition. Each result in the mix must equal the result alone within 1e-9 relative
(max-norm): the arithmetic is the same, only the number of CTAs that reduce the
solver's dot products changes the rounding.
"""
import numpy as np
import pytest

from maze_poisson_b200.c_api import CAPI
from maze_poisson_b200.md import MDRun
from maze_poisson_b200.systems import make_system

pytestmark = pytest.mark.gpu

# (ncell, grid, density, integrator): uneven N (128, 250, 432) and grids (32^3-64^3)
SPECS = [(4, 32, 1.379, "VERLET"), (5, 48, 1.329, "OVRVO"), (6, 64, 1.379, "VERLET")]
STEPS = 6
TOL = 1e-9


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


@pytest.fixture(scope="module")
def prod(product_path):
    return CAPI(product_path)


def new_run(capi, k, spec):
    ncell, n, rho, itg = spec
    h = capi.mzb_system_create()
    run = MDRun(capi, make_system(ncell, n, density=rho, seed=100 + k), method="LCG", tol=1e-10,
                integrator=itg, thermostat=itg == "OVRVO", precision=1)
    run.initialize()
    assert capi.mzb_get_precision() == 1
    return h, run


def test_system_handles(prod):
    h = prod.mzb_system_create()
    assert prod.mzb_system_current() == h
    assert prod.mzb_system_select(h + 1000) == -1
    assert prod.mzb_system_destroy(h) == 0
    assert prod.mzb_system_destroy(h) == -1
    assert prod.mzb_system_footprint(256, 16000) > 10 * 8 * 256 ** 3


def test_batch_matches_alone(prod):
    runs = [new_run(prod, k, spec) for k, spec in enumerate(SPECS)]
    handles = np.array([h for h, _ in runs], dtype=np.int32)
    tuned = np.zeros(4)
    assert prod.mzb_batch_autotune(handles, len(handles), tuned) == 0
    assert 0.0 < tuned[0] <= 1.2 and tuned[1] >= len(SPECS) and tuned[2] > 0 and tuned[3] > 0
    plans = []  # the coarse-level plan the tuner chose for each system's size class
    for h in handles:
        assert prod.mzb_system_select(int(h)) == 0
        plans.append(prod.mzb_get_mixed_plan())
    # the same systems alone, from the same bootstrap, with the same plans
    alone = []
    for k, spec in enumerate(SPECS):
        h, run = new_run(prod, k, spec)
        assert prod.mzb_set_mixed_plan(plans[k]) == 0
        assert prod.mzb_get_mixed_plan() == plans[k]
        for _ in range(STEPS):
            run.step()
        alone.append(run.state(fields=False))
        assert prod.mzb_system_destroy(h) == 0
    launches0 = prod.mzb_kernel_launches()
    assert prod.mzb_batch_step(handles, len(handles), STEPS) == 0
    # each particle stage is one launch over the replica table, whatever the number of
    # systems: about 20 kernels per batched step (the field solves are one of them)
    per_step = (prod.mzb_kernel_launches() - launches0) / STEPS
    assert 0 < per_step <= 24, per_step
    try:
        for (h, run), ref in zip(runs, alone):
            assert prod.mzb_system_select(h) == 0
            st = run.state(fields=False)
            for key in ("pos", "vel", "fcs_tot", "fcs_elec", "fcs_noel"):
                assert rel(st[key], ref[key]) < TOL, (h, key, rel(st[key], ref[key]))
    finally:
        for h, _ in runs:
            prod.mzb_system_destroy(h)


def test_batch_of_one_matches_per_call(prod):
    h0, a = new_run(prod, 0, SPECS[1])
    for _ in range(3):
        a.step()
    ref = a.state(fields=False)
    ocalls = prod.mzb_get_ocalls()
    prod.mzb_system_destroy(h0)
    h1, b = new_run(prod, 0, SPECS[1])
    try:
        assert prod.mzb_batch_step(np.array([h1], dtype=np.int32), 1, 3) == 0
        st = b.state(fields=False)
        assert prod.mzb_get_ocalls() == ocalls  # the Philox counter advanced on the device
        for key in ("pos", "vel", "fcs_tot"):
            assert rel(st[key], ref[key]) < TOL, (key, rel(st[key], ref[key]))
    finally:
        prod.mzb_system_destroy(h1)


def test_classes_match_alone(prod):
    """Size classes side by side (mzb_batch_classes): the 32^3 and 48^3 systems form one
    class on 6 CTAs, the 64^3 system another on 20; over two calls the first class takes
    4 + 2 steps and the second 2 + 1, and each result equals the system stepped alone for
    its own step count."""
    class_of = [0, 0, 1]
    totals = [6, 3]
    alone = []
    for k, spec in enumerate(SPECS):
        h, run = new_run(prod, k, spec)
        for _ in range(totals[class_of[k]]):
            run.step()
        alone.append(run.state(fields=False))
        assert prod.mzb_system_destroy(h) == 0

    runs = [new_run(prod, k, spec) for k, spec in enumerate(SPECS)]
    handles = np.array([h for h, _ in runs], dtype=np.int32)
    cls = np.array(class_of, dtype=np.int32)
    ctas = np.array([6, 20], dtype=np.int32)
    try:
        for steps in ([4, 2], [2, 1]):
            assert prod.mzb_batch_classes(handles, cls, len(handles), ctas, np.array(steps, dtype=np.int32), 2) == 0
        for (h, run), ref in zip(runs, alone):
            assert prod.mzb_system_select(h) == 0
            st = run.state(fields=False)
            for key in ("pos", "vel", "fcs_tot", "fcs_elec", "fcs_noel"):
                assert rel(st[key], ref[key]) < TOL, (h, key, rel(st[key], ref[key]))
    finally:
        for h, _ in runs:
            prod.mzb_system_destroy(h)
