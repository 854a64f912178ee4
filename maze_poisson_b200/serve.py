"""Served form: a request loop that keeps many MD jobs resident on one GPU.

MD jobs (molten-salt systems of uneven size, each with its own step count and
integrator) arrive as a seeded Poisson stream. The loop admits them in arrival order as
slots and device memory free up (the footprint of mzb_system_footprint against an HBM
budget), bootstraps each admitted job through the reference calls (SolverMD.initialize
and initialize_md, maze_poisson/solver.py:96-108, 371-409), keeps its fields and
particle state on the device, and advances all active jobs together in chunks of
mzb_batch_step (continuous batching: membership changes between chunks, never within
one). A job's latency runs from its arrival to the end of its last step.

    python -m maze_poisson_b200.serve --rate 20 --duration 5 --seed 7

prints one JSON line: p50/p99 latency, p50/p99 slowdown against the same job run alone
(from per-configuration step times measured alone), aggregate steps/s, the steps/s of
running the same jobs one after another alone, and occupancy.
With --precision 0 the jobs use the reference's FP64 solvers and are stepped one after
another (solver_md_step), the plain baseline of the served form.
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


class Server:
    """Admission + continuous batching over one library instance (see module doc)."""

    def __init__(self, capi, budget_gb=150.0, max_slots=64, chunk=10, precision=1, tol=1e-10, collect=False):
        self.capi = capi
        self.collect = collect  # keep each job's final positions/velocities/forces
        self.budget = budget_gb * 1e9
        self.max_slots = max_slots
        self.chunk = chunk
        self.precision = precision
        self.tol = tol
        self.active = []
        self.used = 0.0
        self.steps_done = 0
        self.occupancy = []   # active jobs per chunk
        self.autotuned = {}

    def fits(self, job):
        return len(self.active) < self.max_slots and self.used + job.footprint <= self.budget

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

    def advance(self, k):
        c = self.capi
        if self.precision == 1:
            handles = np.array([j.handle for j in self.active], dtype=np.int32)
            # re-tune when the batch's shape (job count to a power of two, largest grid) is new
            key = (1 << len(self.active).bit_length(), max(j.n_grid for j in self.active))
            if key not in self.autotuned and len(self.active) > 1:
                out = np.zeros(4)
                c.mzb_batch_autotune(handles, len(handles), out)
                self.autotuned[key] = out.tolist()
            if c.mzb_batch_step(handles, len(handles), k) != 0:
                raise RuntimeError("a field solve did not converge")
        else:
            for j in self.active:
                c.mzb_system_select(j.handle)
                c.solver_md_step(k)
        for j in self.active:
            j.done += k
        self.steps_done += k * len(self.active)
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
            while pending and pending[0].arrival <= now and self.fits(pending[0]):
                self.admit(pending.pop(0), time.perf_counter() - t0)
            if not self.active:
                time.sleep(max(0.0, min(pending[0].arrival - now, 0.05)))
                continue
            k = min(self.chunk, min(j.steps - j.done for j in self.active))
            self.advance(k)
            now = time.perf_counter() - t0
            for j in [j for j in self.active if j.done >= j.steps]:
                self.retire(j, now)
        return jobs


def isolated_step_times(capi, jobs, precision, tol, steps=5):
    """Per (grid, ncell, integrator): seconds of the bootstrap and of one step, the job
    alone on the GPU through the same calls the loop makes."""
    out = {}
    for key in sorted({(j.n_grid, j.ncell, j.integrator) for j in jobs}):
        n_grid, ncell, itg = key
        job = Job(jid=-1, arrival=0, ncell=ncell, n_grid=n_grid, density=1.35, steps=steps,
                  integrator=itg, seed=1)
        h = capi.mzb_system_create()
        run = make_run(capi, job, precision, tol)
        t0 = time.perf_counter()
        run.initialize()
        t1 = time.perf_counter()
        hs = np.array([h], dtype=np.int32)
        if precision == 1:
            capi.mzb_batch_step(hs, 1, 3)  # the three step graphs of this system
            t1b = time.perf_counter()
            capi.mzb_batch_step(hs, 1, steps)
        else:
            capi.solver_md_step(1)
            t1b = time.perf_counter()
            capi.solver_md_step(steps)
        t2 = time.perf_counter()
        capi.mzb_system_destroy(h)
        out[key] = (t1 - t0, (t2 - t1b) / steps)  # the warm-up steps are in neither
    return out


def summarize(jobs, server, iso, wall):
    lat = np.array([j.finished - j.arrival for j in jobs])
    alone = np.array([iso[(j.n_grid, j.ncell, j.integrator)][0] + j.steps * iso[(j.n_grid, j.ncell, j.integrator)][1]
                      for j in jobs])
    slow = lat / alone
    total_steps = sum(j.steps for j in jobs)
    return {
        "sequential_alone_steps_per_s": total_steps / float(alone.sum()),
        "jobs": len(jobs),
        "p50_latency_s": float(np.percentile(lat, 50)), "p99_latency_s": float(np.percentile(lat, 99)),
        "p50_slowdown_vs_alone": float(np.percentile(slow, 50)),
        "p99_slowdown_vs_alone": float(np.percentile(slow, 99)),
        "steps_per_s": total_steps / wall, "job_steps": total_steps, "wall_s": wall,
        "mean_active_jobs": float(np.mean(server.occupancy)) if server.occupancy else 0.0,
        "max_active_jobs": int(max(server.occupancy)) if server.occupancy else 0,
    }


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
    ap.add_argument("--chunk", type=int, default=10)
    ap.add_argument("--precision", type=int, default=1, choices=[0, 1])
    ap.add_argument("--tol", type=float, default=1e-10)
    args = ap.parse_args()
    os.environ.setdefault("MZB_QUIET", "1")
    capi = CAPI()
    jobs = job_stream(args.seed, args.rate, args.duration, args.n_min, args.n_max,
                      (args.steps_min, args.steps_max))
    server = Server(capi, args.budget_gb, args.slots, args.chunk, args.precision, args.tol)
    t0 = time.perf_counter()
    server.serve(jobs)
    wall = time.perf_counter() - t0
    iso = isolated_step_times(capi, jobs, args.precision, args.tol)
    line = {"form": "served", "precision": "fp32_refine" if args.precision else "fp64",
            "rate_per_s": args.rate, "arrival_window_s": args.duration, "seed": args.seed,
            "budget_gb": args.budget_gb, "slots": args.slots, "chunk": args.chunk,
            **summarize(jobs, server, iso, wall),
            "autotuned": {str(k): v for k, v in list(server.autotuned.items())[:4]}}
    print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
