"""Served form (maze_poisson_b200/serve.py): a short Poisson stream of uneven jobs is
admitted against a memory budget and advanced by continuous batching, with the jobs side
by side on their own SM shares (policy shared) or in one lockstep batch; every job
finishes, and the results of jobs that ran in the mix equal the same jobs run alone
through the per-call reference path within 1e-9 relative (max-norm)."""
import numpy as np
import pytest

from maze_poisson_b200.c_api import CAPI
from maze_poisson_b200.serve import Server, calibrate, job_stream, make_run

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


@pytest.fixture(scope="module")
def prod(product_path):
    return CAPI(product_path)


@pytest.mark.parametrize("policy", ["shared", "lockstep"])
def test_served_stream_matches_alone(prod, policy):
    jobs = job_stream(seed=3, rate=200.0, duration=0.03, n_min=128, n_max=700, steps=(4, 13))
    assert len(jobs) >= 3
    costs = calibrate(prod, {j.key for j in jobs}, 1, 1e-10, steps=2)
    assert all(c.alone > 0 and c.boot > 0 for c in costs.values())
    # a budget that holds only part of the stream at once, so admission waits for retirements;
    # a slowdown bound that admits every job that fits
    budget = 1e-9 * sum(prod.mzb_system_footprint(j.n_grid, j.n_ions) for j in jobs) * 0.6
    server = Server(prod, costs, budget_gb=budget, max_slots=4, chunk=3, precision=1, tol=1e-10,
                    policy=policy, beta=1e9, call_ms=5.0, collect=True)
    server.serve(jobs)
    assert all(j.done == j.steps and j.finished >= j.admitted >= j.arrival for j in jobs)
    assert max(server.occupancy) >= 2
    for job in jobs[:3]:
        h = prod.mzb_system_create()
        run = make_run(prod, job, 1, 1e-10)
        run.initialize()
        for _ in range(job.steps):
            run.step()
        alone = run.state(fields=False)
        prod.mzb_system_destroy(h)
        for key in ("pos", "vel", "fcs_tot"):
            assert rel(job.final[key], alone[key]) < 1e-9, (job.jid, key, rel(job.final[key], alone[key]))
