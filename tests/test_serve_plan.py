"""Host logic of the served form (no GPU): the step-time model t(c) = a + b / c of a job
on c CTAs, the water-filled CTA shares and the slowdown-bounded admission."""
import math

import pytest

from maze_poisson_b200.serve import Cost, Job, Server, fit_cost, plan_shares

SMS = 148
# fitted on a B200 (seconds per MD step): 64^3 / 250 ions and 256^3 / 16000 ions
SMALL = Cost(boot=0.03, a=0.82e-3, b=14.7e-3, sms=SMS)
BIG = Cost(boot=0.05, a=3.3e-3, b=276e-3, sms=SMS)


class FakeLibrary:
    def mzb_sm_count(self):
        return SMS


def test_fit_cost_recovers_model():
    c = fit_cost(0.1, BIG.step(SMS), BIG.step(12), SMS, 12)
    assert math.isclose(c.a, BIG.a, rel_tol=1e-9) and math.isclose(c.b, BIG.b, rel_tol=1e-9)
    flat = fit_cost(0.1, 2e-3, 1.9e-3, SMS, 12)  # noise: fewer CTAs measured faster
    assert flat.b == 0.0 and flat.a == 2e-3 and flat.ctas_for(1.0) == 1


def test_ctas_for_is_the_fewest():
    for sd in (1.2, 1.5, 2.0, 4.0):
        c = BIG.ctas_for(sd)
        assert BIG.step(c) <= sd * BIG.alone + 1e-15
        assert c == 1 or BIG.step(c - 1) > sd * BIG.alone
    assert SMALL.ctas_for(1.0) == SMS and SMALL.ctas_for(0.9) is None


@pytest.mark.parametrize("mix", [[SMALL], [BIG], [BIG, BIG], [BIG] + [SMALL] * 6, [SMALL] * 40, [BIG] * 148])
def test_plan_shares(mix):
    sd, shares = plan_shares(mix, SMS)
    assert sum(shares) == SMS and min(shares) >= 1
    assert all(math.isclose(s, c.step(n) / c.alone) for s, c, n in zip(sd, mix, shares))
    # no single CTA moved from a faster job to the slowest one lowers the largest slowdown
    worst = max(range(len(mix)), key=lambda i: sd[i])
    for i in range(len(mix)):
        if i != worst and shares[i] > 1:
            moved = list(shares)
            moved[i] -= 1
            moved[worst] += 1
            after = [c.step(n) / c.alone for c, n in zip(mix, moved)]
            assert max(after) >= max(sd) - 1e-12
    if len(mix) == 1:
        assert shares == [SMS] and math.isclose(sd[0], 1.0)


def test_plan_shares_limits():
    assert plan_shares([], SMS) == ([], [])
    assert plan_shares([SMALL] * (SMS + 1), SMS) == (None, None)


def job(jid, cost_key):
    ncell, grid = cost_key
    j = Job(jid=jid, arrival=0.0, ncell=ncell, n_grid=grid, density=1.35, steps=100, integrator="VERLET", seed=1)
    j.footprint = 1e9
    return j


def test_admission_bounded_by_predicted_slowdown():
    costs = {(64, 5): SMALL, (256, 20): BIG}
    server = Server(FakeLibrary(), costs, budget_gb=150.0, max_slots=64, beta=1.8)
    server.interference = 1.0
    admitted = []
    for k in range(64):
        j = job(k, (5, 64) if k % 4 else (20, 256))
        if not server.fits(j):
            break
        server.active.append(j)  # admitted without a library call
        server.used += j.footprint
        admitted.append(j)
    assert len(admitted) >= 2
    sd, _ = plan_shares([costs[j.key] for j in server.active], SMS)
    assert max(sd) <= 1.8
    # the job refused would have pushed some job past the bound
    nxt = job(99, (5, 64) if len(admitted) % 4 else (20, 256))
    sd2, _ = plan_shares([costs[j.key] for j in server.active + [nxt]], SMS)
    assert sd2 is None or max(sd2) > 1.8
    # the measured interference tightens the bound
    server.interference = 2.0
    assert not server.fits(job(100, (5, 64)))
    # slots and memory still bound every policy
    lock = Server(FakeLibrary(), costs, budget_gb=2.5, max_slots=64, policy="lockstep")
    lock.active, lock.used = [job(0, (5, 64)), job(1, (5, 64))], 2e9
    assert not lock.fits(job(2, (5, 64)))


def test_plan_steps_follow_pace():
    costs = {(64, 5): SMALL, (256, 20): BIG}
    server = Server(FakeLibrary(), costs, call_ms=25.0)
    server.active = [job(0, (20, 256)), job(1, (5, 64)), job(2, (5, 64))]
    server.active[2].done = 97  # three steps left
    sd, shares, steps, expect = server.plan()
    assert sum(shares) == SMS
    t = [costs[j.key].step(s) for j, s in zip(server.active, shares)]
    assert steps[2] == 3
    assert steps[1] >= 10 * steps[0] // 2  # the small job takes many steps per call
    assert math.isclose(expect, max(n * x for n, x in zip(steps, t)))
