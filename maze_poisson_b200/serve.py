"""Served form: a request loop that keeps many MD jobs resident on one GPU.

MD jobs (molten-salt systems of uneven size, each with its own step count and
integrator) arrive as a seeded Poisson stream. The loop admits them in arrival order as
slots and device memory free up (the footprint of mzb_system_footprint against an HBM
budget), bootstraps each admitted job through the reference calls (SolverMD.initialize
and initialize_md, maze_poisson/solver.py:96-108, 371-409), keeps its fields and
particle state on the device, and advances the active jobs together in calls of the
batched step (continuous batching: membership changes between calls, never within one).

Two policies:

* ``shared`` (default): every active job is its own class of mzb_batch_classes, with its
  own stream and its own share of the SMs for its cooperative field solve, so jobs of
  different sizes run side by side, each at its own pace. A calibrated cost model gives
  each job's step time on c CTAs, t(c) = a + b / c (a: latency-bound part, b: the part
  that scales with the SMs), fitted from two timed runs of the job's configuration alone.
  The shares are water-filled to equalise the predicted slowdown t(c_j) / t(all SMs)
  across jobs, and a job is admitted only while the predicted slowdown of every active
  job, times the measured interference factor of recent calls, stays within ``beta``.
  Each call gives job j about ``call_ms`` / t(c_j) steps.
* ``lockstep``: all active jobs in ONE batched step per MD step (mzb_batch_step after
  mzb_batch_autotune), admitted by slots and memory only; every job moves at the pace of
  the slowest.

A job's latency runs from its admission to the end of its last step (its bootstrap
included); the queueing wait before admission is reported on its own. The slowdown of a
job is its latency over the same job run alone on the whole GPU (bootstrap + steps x its
step time alone, from the calibration).

    python -m maze_poisson_b200.serve --rate 20 --duration 5 --seed 7

prints one JSON line. With --precision 0 the jobs use the reference's FP64 solvers and
are stepped one after another in chunks (solver_md_step), the plain baseline.
"""
import argparse
import dataclasses
import json
import math
import os
import time

import numpy as np

from .c_api import CAPI
from .md import MDRun
from .systems import box_length_ang, make_system

GRIDS = (64, 96, 128, 160, 192, 224, 256)  # even, coarsened at least three times


@dataclasses.dataclass
class Job:
    jid: int
    arrival: float        # s after the start
    ncell: int            # N = 2 ncell^3
    n_grid: int
    density: float
    steps: int
    integrator: str
    seed: int
    handle: int = -1
    run: object = None
    done: int = 0
    admitted: float = math.nan
    finished: float = math.nan
    footprint: float = 0.0
    final: object = None

    @property
    def n_ions(self):
        return 2 * self.ncell ** 3

    @property
    def key(self):
        return (self.n_grid, self.ncell)


def grid_for(n_ions, density, spacing_ang=0.3):
    """The allowed grid closest to a spacing of `spacing_ang` for this box."""
    target = box_length_ang(n_ions, density) / spacing_ang
    return min(GRIDS, key=lambda g: abs(g - target))


def job_stream(seed, rate, duration, n_min=250, n_max=16000, steps=(50, 500),
               density=(1.30, 1.40), integrators=("VERLET", "OVRVO")):
    """Poisson arrivals (mean `rate` per s) over `duration` s: N log-uniform in
    [n_min, n_max] (as 2 ncell^3), density uniform, grid at ~0.3 A, steps uniform,
    integrator uniform."""
    rng = np.random.default_rng(seed)
    jobs, t = [], 0.0
    lo, hi = math.log(n_min), math.log(n_max)
    while True:
        t += rng.exponential(1.0 / rate)
        if t > duration:
            break
        n = math.exp(rng.uniform(lo, hi))
        ncell = int(round((n / 2) ** (1.0 / 3.0)))
        ncell = max(2, ncell)
        rho = float(rng.uniform(*density))
        jobs.append(Job(jid=len(jobs), arrival=t, ncell=ncell, n_grid=grid_for(2 * ncell ** 3, rho),
                        density=rho, steps=int(rng.integers(steps[0], steps[1] + 1)),
                        integrator=str(rng.choice(integrators)), seed=int(rng.integers(1 << 30))))
    return jobs


def make_run(capi, job, precision, tol):
    system = make_system(job.ncell, job.n_grid, density=job.density, seed=job.seed)
    return MDRun(capi, system, method="LCG", tol=tol, integrator=job.integrator,
                 thermostat=job.integrator == "OVRVO", precision=precision)


# -- cost model and CTA shares ---------------------------------------------------------

@dataclasses.dataclass
class Cost:
    """Seconds: bootstrap, and one MD step on c CTAs, t(c) = a + b / c."""
    boot: float
    a: float
    b: float
    sms: int

    @property
    def alone(self):
        return self.step(self.sms)

    def step(self, ctas):
        return self.a + self.b / ctas

    def ctas_for(self, slowdown):
        """Fewest CTAs with t(c) <= slowdown x t(all SMs), or None if none is enough."""
        room = slowdown * self.alone - self.a
        if self.b <= 0:  # no part that scales with the SMs
            return 1 if room >= -1e-15 * self.a else None
        if room <= 0:
            return None
        c = max(1, math.ceil(self.b / room - 1e-12))
        return c if c <= self.sms else None


def fit_cost(boot, t_all, t_low, sms, low):
    """a, b of t(c) = a + b / c through (sms, t_all) and (low, t_low), b >= 0, a >= 0."""
    b = max(0.0, (t_low - t_all) / (1.0 / low - 1.0 / sms))
    a = max(0.0, t_all - b / sms)
    return Cost(boot=boot, a=a, b=b, sms=sms)


def plan_shares(costs, sms):
    """CTA shares that minimise the largest predicted slowdown t(c_j) / t(sms): bisection
    on the slowdown for the fewest CTAs each job needs, then leftover CTAs one at a time to
    the job that is slowest. Returns (predicted slowdowns, shares), or (None, None) when
    the jobs need more than one CTA each than there are SMs."""
    n = len(costs)
    if n == 0:
        return [], []
    if n > sms:
        return None, None

    def need(sd):
        cs = [c.ctas_for(sd) for c in costs]
        return None if any(c is None for c in cs) else cs

    lo, hi = 1.0, 2.0
    while need(hi) is None or sum(need(hi)) > sms:
        hi *= 2.0
        if hi > 1e7:
            return None, None
    for _ in range(60):
        mid = 0.5 * (lo + hi)
        cs = need(mid)
        if cs is not None and sum(cs) <= sms:
            hi = mid
        else:
            lo = mid
    shares = need(hi)
    left = sms - sum(shares)
    while left > 0:
        j = max(range(n), key=lambda i: costs[i].step(shares[i]) / costs[i].alone)
        shares[j] += 1
        left -= 1
    return [c.step(s) / c.alone for c, s in zip(costs, shares)], shares


def calibrate(capi, keys, precision, tol, steps=6, low=12):
    """Cost per (grid, ncell): each configuration alone on the GPU, bootstrapped through
    the same calls the loop makes, then timed on all SMs and (FP32+refine) on `low` CTAs.
    The first system only warms up the library."""
    sms = capi.mzb_sm_count()
    out = {}
    order = [min(keys)] + sorted(keys)
    for i, key in enumerate(order):
        n_grid, ncell = key
        job = Job(jid=-1, arrival=0, ncell=ncell, n_grid=n_grid, density=1.35, steps=steps,
                  integrator="VERLET", seed=1)
        h = capi.mzb_system_create()
        run = make_run(capi, job, precision, tol)
        t0 = time.perf_counter()
        run.initialize()
        boot = time.perf_counter() - t0
        if precision == 1:
            hs, cls, one = (np.array([h], dtype=np.int32), np.zeros(1, dtype=np.int32),
                            np.ones(1, dtype=np.int32))
            timed = []
            for ctas in (sms, low):
                c = np.array([ctas], dtype=np.int32)
                capi.mzb_batch_classes(hs, cls, 1, c, 3 * one, 1)  # the three graphs of this share
                t1 = time.perf_counter()
                capi.mzb_batch_classes(hs, cls, 1, c, steps * one, 1)
                timed.append((time.perf_counter() - t1) / steps)
            cost = fit_cost(boot, timed[0], timed[1], sms, low)
        else:
            capi.solver_md_step(1)
            t1 = time.perf_counter()
            capi.solver_md_step(steps)
            t_all = (time.perf_counter() - t1) / steps
            cost = Cost(boot=boot, a=t_all, b=0.0, sms=sms)
        capi.mzb_system_destroy(h)
        if i > 0:
            out[key] = cost
    return out


# -- the loop --------------------------------------------------------------------------

class Server:
    """Admission + continuous batching over one library instance (see module doc)."""

    def __init__(self, capi, costs=None, budget_gb=150.0, max_slots=64, chunk=10, precision=1, tol=1e-10,
                 policy="shared", beta=1.5, call_ms=25.0, admit_per_call=1, collect=False):
        self.capi = capi
        self.costs = costs or {}
        self.collect = collect  # keep each job's final positions/velocities/forces
        self.budget = budget_gb * 1e9
        self.max_slots = max_slots
        self.chunk = chunk
        self.precision = precision
        self.tol = tol
        self.policy = policy if precision == 1 else "sequential"
        self.beta = beta
        self.call_s = call_ms * 1e-3
        # bootstraps run between calls and stall every active job: at most this many per
        # call (0 = no limit), so that a job admitted starts stepping promptly
        self.admit_per_call = admit_per_call
        self.sms = capi.mzb_sm_count()
        self.interference = 1.0  # measured call time / predicted, smoothed over calls
        self.active = []
        self.used = 0.0
        self.steps_done = 0
        self.occupancy = []      # active jobs per call
        self.queued = []         # jobs waiting for admission per call
        self.predicted = []      # largest predicted slowdown per call
        self.autotuned = {}
        self.seconds = {"calls": 0.0, "admit": 0.0, "retire": 0.0, "plan": 0.0}

    def cost(self, job):
        if job.key not in self.costs:
            raise KeyError(f"no calibrated cost for grid {job.n_grid}, ncell {job.ncell}")
        return self.costs[job.key]

    def fits(self, job):
        if len(self.active) >= self.max_slots or self.used + job.footprint > self.budget:
            return False
        if self.policy != "shared" or not self.active:
            return True
        sd, _ = plan_shares([self.cost(j) for j in self.active + [job]], self.sms)
        return sd is not None and max(sd) * self.interference <= self.beta

    def admit(self, job, now):
        c = self.capi
        job.handle = c.mzb_system_create()
        job.run = make_run(c, job, self.precision, self.tol)
        job.run.initialize()
        job.admitted = now
        self.active.append(job)
        self.used += job.footprint

    def retire(self, job, now):
        job.finished = now
        if self.collect:
            self.capi.mzb_system_select(job.handle)
            job.final = job.run.state(fields=False)
        self.capi.mzb_system_destroy(job.handle)
        job.run = None
        self.active.remove(job)
        self.used -= job.footprint

    def plan(self):
        """Shares and step counts of the next call (policy shared)."""
        costs = [self.cost(j) for j in self.active]
        sd, shares = plan_shares(costs, self.sms)
        if sd is None:
            raise RuntimeError("more active jobs than SMs")
        times = [c.step(s) for c, s in zip(costs, shares)]
        span = max(self.call_s, 2.0 * max(times))
        steps = [max(1, min(j.steps - j.done, int(round(span / t)))) for j, t in zip(self.active, times)]
        return sd, shares, steps, max(n * t for n, t in zip(steps, times))

    def advance(self):
        c = self.capi
        handles = np.array([j.handle for j in self.active], dtype=np.int32)
        t0 = time.perf_counter()
        if self.policy == "shared":
            sd, shares, steps, expect = self.plan()
            t1 = time.perf_counter()
            self.seconds["plan"] += t1 - t0
            rc = c.mzb_batch_classes(handles, np.arange(len(handles), dtype=np.int32), len(handles),
                                     np.array(shares, dtype=np.int32), np.array(steps, dtype=np.int32),
                                     len(handles))
            wall = time.perf_counter() - t1
            self.interference = 0.7 * self.interference + 0.3 * max(1.0, wall / expect)
            self.predicted.append(max(sd))
        elif self.policy == "lockstep":
            k = min(self.chunk, min(j.steps - j.done for j in self.active))
            key = (1 << len(self.active).bit_length(), max(j.n_grid for j in self.active))
            if key not in self.autotuned and len(self.active) > 1:
                out = np.zeros(4)
                c.mzb_batch_autotune(handles, len(handles), out)
                self.autotuned[key] = out.tolist()
            rc = c.mzb_batch_step(handles, len(handles), k)
            steps = [k] * len(self.active)
        else:
            k = min(self.chunk, min(j.steps - j.done for j in self.active))
            rc = 0
            for j in self.active:
                c.mzb_system_select(j.handle)
                c.solver_md_step(k)
            steps = [k] * len(self.active)
        self.seconds["calls"] += time.perf_counter() - t0
        if rc != 0:
            raise RuntimeError("a field solve did not converge")
        for j, k in zip(self.active, steps):
            j.done += k
        self.steps_done += sum(steps)
        self.occupancy.append(len(self.active))

    def serve(self, jobs):
        """Run the stream in real time; returns the jobs with their timestamps."""
        for j in jobs:
            j.footprint = self.capi.mzb_system_footprint(j.n_grid, j.n_ions)
            if j.footprint > self.budget:
                raise ValueError(f"job {j.jid} needs {j.footprint / 1e9:.1f} GB, more than the budget")
        pending = sorted(jobs, key=lambda j: j.arrival)
        t0 = time.perf_counter()
        while pending or self.active:
            now = time.perf_counter() - t0
            ta = time.perf_counter()
            n_adm = 0
            while (pending and pending[0].arrival <= now and self.fits(pending[0])
                   and (self.admit_per_call <= 0 or n_adm < self.admit_per_call)):
                self.admit(pending.pop(0), time.perf_counter() - t0)
                n_adm += 1
            self.seconds["admit"] += time.perf_counter() - ta
            if not self.active:
                time.sleep(max(0.0, min(pending[0].arrival - now, 0.05)))
                continue
            self.queued.append(sum(1 for j in pending if j.arrival <= now))
            self.advance()
            now = time.perf_counter() - t0
            tr = time.perf_counter()
            for j in [j for j in self.active if j.done >= j.steps]:
                self.retire(j, now)
            self.seconds["retire"] += time.perf_counter() - tr
        return jobs


def summarize(jobs, server, costs, wall):
    lat = np.array([j.finished - j.admitted for j in jobs])
    lat_q = np.array([j.finished - j.arrival for j in jobs])
    alone = np.array([costs[j.key].boot + j.steps * costs[j.key].alone for j in jobs])
    slow = lat / alone
    total_steps = sum(j.steps for j in jobs)
    occ = np.array(server.occupancy) if server.occupancy else np.zeros(1)
    queued = np.array(server.queued) if server.queued else np.zeros(1)
    return {
        "jobs": len(jobs), "job_steps": total_steps, "wall_s": wall,
        "steps_per_s": total_steps / wall,
        "sequential_alone_steps_per_s": total_steps / float(alone.sum()),
        "p50_latency_s": float(np.percentile(lat, 50)), "p99_latency_s": float(np.percentile(lat, 99)),
        "p50_slowdown_vs_alone": float(np.percentile(slow, 50)),
        "p99_slowdown_vs_alone": float(np.percentile(slow, 99)),
        "max_slowdown_vs_alone": float(slow.max()),
        "p50_latency_with_queue_s": float(np.percentile(lat_q, 50)),
        "p99_latency_with_queue_s": float(np.percentile(lat_q, 99)),
        "mean_active_jobs": float(occ.mean()), "max_active_jobs": int(occ.max()),
        "calls_with_jobs_waiting": float(np.mean(queued > 0)),
        "latency_from": "admission (bootstrap included); queueing reported apart",
        "calls": len(server.occupancy),
        "seconds_in": {k: round(v, 3) for k, v in server.seconds.items()},
    }


def job_records(jobs, costs):
    """Per job: configuration, timestamps, time alone and slowdown."""
    out = []
    for j in jobs:
        alone = costs[j.key].boot + j.steps * costs[j.key].alone
        out.append({"jid": j.jid, "grid": j.n_grid, "n_ions": j.n_ions, "steps": j.steps,
                    "integrator": j.integrator, "arrival": j.arrival, "admitted": j.admitted,
                    "finished": j.finished, "boot_alone_s": costs[j.key].boot, "alone_s": alone,
                    "slowdown": (j.finished - j.admitted) / alone})
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--rate", type=float, default=20.0, help="mean arrivals per second")
    ap.add_argument("--duration", type=float, default=5.0, help="seconds of arrivals")
    ap.add_argument("--seed", type=int, default=7)
    ap.add_argument("--n-min", type=int, default=250)
    ap.add_argument("--n-max", type=int, default=16000)
    ap.add_argument("--steps-min", type=int, default=50)
    ap.add_argument("--steps-max", type=int, default=500)
    ap.add_argument("--budget-gb", type=float, default=150.0)
    ap.add_argument("--slots", type=int, default=64)
    ap.add_argument("--chunk", type=int, default=10, help="steps per call (lockstep, sequential)")
    ap.add_argument("--precision", type=int, default=1, choices=[0, 1])
    ap.add_argument("--tol", type=float, default=1e-10)
    ap.add_argument("--policy", default="shared", choices=["shared", "lockstep"])
    ap.add_argument("--beta", type=float, default=1.5, help="admission bound on predicted slowdown (shared)")
    ap.add_argument("--call-ms", type=float, default=25.0, help="target length of one call (shared)")
    ap.add_argument("--admit-per-call", type=int, default=1, help="bootstraps between two calls (0: no limit)")
    ap.add_argument("--jobs-out", default=None, help="write per-job records (JSON) to this file")
    args = ap.parse_args()
    os.environ.setdefault("MZB_QUIET", "1")
    capi = CAPI()
    jobs = job_stream(args.seed, args.rate, args.duration, args.n_min, args.n_max,
                      (args.steps_min, args.steps_max))
    t0 = time.perf_counter()
    costs = calibrate(capi, {j.key for j in jobs}, args.precision, args.tol)
    calib_s = time.perf_counter() - t0
    server = Server(capi, costs, args.budget_gb, args.slots, args.chunk, args.precision, args.tol,
                    policy=args.policy, beta=args.beta, call_ms=args.call_ms, admit_per_call=args.admit_per_call)
    t0 = time.perf_counter()
    server.serve(jobs)
    wall = time.perf_counter() - t0
    line = {"form": "served", "precision": "fp32_refine" if args.precision else "fp64",
            "policy": server.policy, "beta": args.beta if server.policy == "shared" else None,
            "call_ms": args.call_ms, "admit_per_call": args.admit_per_call,
            "rate_per_s": args.rate, "arrival_window_s": args.duration, "seed": args.seed,
            "budget_gb": args.budget_gb, "slots": args.slots, "calibration_s": calib_s,
            **summarize(jobs, server, costs, wall),
            "mean_predicted_slowdown": float(np.mean(server.predicted)) if server.predicted else None,
            "interference": server.interference}
    print(json.dumps(line), flush=True)
    if args.jobs_out:
        with open(args.jobs_out, "w") as f:
            json.dump(job_records(jobs, costs), f)


if __name__ == "__main__":
    main()
