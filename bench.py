#!/usr/bin/env python
"""Benchmark of the MaZe_Poisson MD hot path on B200 (one JSON line on rank 0).

Workload (the reference's configuration 1): 2000 Na+/Cl- ions at 1.329 g/cm^3 on a
10^3-cell lattice with +-0.1a jitter and 1200 K Maxwell-Boltzmann velocities; 128^3 grid,
CIC spreading, LCG (CG with implicit Jacobi) at tol 1e-8, Tosi-Fumi forces with
r_cut = L/2, OVRVO Langevin at 1200 K with friction 1 ps^-1, dt = 1 fs. Synthetic, seeded.

A step is one SolverMD.md_loop_iter (maze_poisson/solver.py:483-492): integrator part 1,
charge spreading, field solve, field + pair + total forces, integrator part 2.

  value : steps/s with the state resident on the GPU, each step run by solver_md_step(1)
          and timed with CUDA events on the library's stream; L2 (126 MB) is flushed by
          writing a 256 MB buffer on that stream before every timed step (outside the
          events). N GPUs run N independent replicas (weak scaling); the job's value is
          total steps / max-over-ranks time.
  e2e   : steps/s of a whole job through the reference's ctypes ABI from host buffers:
          solver_initialize_particles (H2D from pinned host memory), the two bootstrap
          steps, then K steps of the reference's per-call sequence, each followed by the
          output getters get_pos/get_vel/get_fcs_tot (D2H into pinned host memory);
          wall-clock over the whole job / K.
  modes : the same steps with the field solve in FP32 multigrid + FP64 refinement
          (same FP64 residual tolerance), its steps/s and force RMS error against FP64.
  roofline : the solver-engine launch (one field solve per step) against the measured
          HBM copy bandwidth; algorithmic bytes per launch = (5 + 8 (it+1)) * 8 B * n^3
          (CG: x, r, p read+write and Ap write+read per iteration; set-up 5 passes).

`--impl reference` times the reference's own C library (built from its sources, shipped
Release flags, OpenMP on every host core) through its facade on the same workload.
"""
import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "MD steps/s (FP64 LCG; configuration nacl2000_128)"
WORKLOAD = dict(ncell=10, n_grid=128, density=1.329)
SOLVER = dict(method="LCG", precond="NONE", tol=1e-8, integrator="OVRVO", thermostat=True, T=1200.0,
              gamma_per_ps=1.0, dt_fs=1.0)
CONFIG = {"workload": "nacl2000_128", "n_ions": 2000, "grid": 128, "density_g_cm3": 1.329,
          "method": "LCG", "tol": 1e-8, "integrator": "OVRVO", "T_K": 1200, "gamma_per_ps": 1.0,
          "dt_fs": 1.0, "l2": "flushed (256 MB write) before every timed step",
          "parallelism": "replicas"}


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def load_traffic():
    """Per-launch DRAM bytes of the solver engine from a committed ncu summary, if any."""
    try:
        with open(os.path.join(ROOT, "profiles", "engine_traffic.json")) as f:
            return json.load(f)
    except Exception:
        return None


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = max(mx, float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        os.unlink(self.path)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def make_run(capi, rank, precision=0):
    from maze_poisson_b200.md import MDRun
    from maze_poisson_b200.systems import make_system
    system = make_system(seed=1000 + rank, T=SOLVER["T"], **WORKLOAD)
    return MDRun(capi, system, precision=precision, **{k: v for k, v in SOLVER.items()})


def timed_steps(capi, stream, flush, steps):
    """Device time of `steps` MD steps (CUDA events on the library stream, L2 flushed
    before each), the mean solve time and the solver's return values."""
    import torch
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    solve_ms, iters = [], []
    for k in range(steps):
        with torch.cuda.stream(stream):
            flush.fill_(float(k))
            ev[k][0].record(stream)
        capi.solver_md_step(1)
        with torch.cuda.stream(stream):
            ev[k][1].record(stream)
        solve_ms.append(capi.mzb_last_solve_ms())
        iters.append(capi.mzb_last_solve_result())
    torch.cuda.synchronize()
    return sum(a.elapsed_time(b) for a, b in ev), solve_ms, iters


def bench_b200(args, rank, world, dist):
    import numpy as np
    import torch

    local = int(os.environ.get("LOCAL_RANK", "0"))
    os.environ["MZB_DEVICE"] = str(local)
    os.environ.setdefault("MZB_QUIET", "1")
    torch.cuda.set_device(local)
    from maze_poisson_b200.c_api import CAPI
    capi = CAPI()
    run = make_run(capi, rank)
    run.initialize()
    stream = torch.cuda.ExternalStream(capi.mzb_get_stream(), device=local)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=f"cuda:{local}")
    for _ in range(args.warmup):
        capi.solver_md_step(1)
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    launches0 = capi.mzb_kernel_launches()
    total_ms, solve_ms, iters = timed_steps(capi, stream, flush, args.steps)
    launches = capi.mzb_kernel_launches() - launches0
    clk = clocks.stop()
    t = torch.tensor([total_ms], dtype=torch.float64, device=f"cuda:{local}")
    if dist is not None:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    max_ms = float(t.item())
    run.finalize()

    # FP32+refine form on the same workload and tolerance: steps/s and its force error
    # against the FP64 form at the same initial state (after the two bootstrap steps)
    mixed = None
    if not args.fp64_only:
        ref = make_run(capi, rank)
        ref.initialize()
        f_ref = ref.state(fields=False)["fcs_tot"]
        ref.finalize()
        mrun = make_run(capi, rank, precision=1)
        mrun.initialize()
        f_mix = mrun.state(fields=False)["fcs_tot"]
        stream = torch.cuda.ExternalStream(capi.mzb_get_stream(), device=local)
        for _ in range(args.warmup):
            capi.solver_md_step(1)
        torch.cuda.synchronize()
        m_ms, m_solve, m_iters = timed_steps(capi, stream, flush, args.steps)
        mrun.finalize()
        tm = torch.tensor([m_ms], dtype=torch.float64, device=f"cuda:{local}")
        if dist is not None:
            dist.all_reduce(tm, op=dist.ReduceOp.MAX)
        rms = float(np.sqrt(np.mean((f_mix - f_ref) ** 2)) / np.sqrt(np.mean(f_ref ** 2)))
        mixed = {"value": round(args.steps * world / (float(tm.item()) / 1e3), 3), "unit": "steps/s",
                 "ms_per_step": round(float(tm.item()) / args.steps, 4),
                 "solve_ms": round(statistics.mean(m_solve), 4),
                 "refinement_steps": statistics.mean(m_iters),
                 "force_rms_rel_err_vs_fp64": rms,
                 "dtype": "f32 multigrid + f64 refinement"}
    del flush
    # end to end through the reference ABI from pinned host buffers
    e2e = bench_e2e(args, capi, rank)
    if dist is not None:
        et = torch.tensor([e2e["seconds"]], dtype=torch.float64, device=f"cuda:{local}")
        dist.all_reduce(et, op=dist.ReduceOp.MAX)
        e2e["seconds"] = float(et.item())

    n3 = WORKLOAD["n_grid"] ** 3
    mean_solve_s = statistics.mean(solve_ms) / 1e3
    mean_iters = statistics.mean(i + 1 for i in iters)
    alg_bytes = (5 + 8 * mean_iters) * 8 * n3
    peak, peak_kind = load_peaks()
    achieved = alg_bytes / mean_solve_s / 1e9
    traffic = load_traffic()
    line = {
        "metric": METRIC,
        "value": round(args.steps * world / (max_ms / 1e3), 3),
        "unit": "steps/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(max_ms / args.steps, 4),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic (seeded NaCl lattice, jitter 0.1a, MB velocities)",
        "config": CONFIG,
        "e2e": {"value": round(args.steps * world / e2e["seconds"], 3), "unit": "steps/s",
                "h2d_bytes_per_step": e2e["h2d"], "d2h_bytes_per_step": e2e["d2h"]},
        "roofline": {"kernel": "engine_kernel (LCG field solve)", "bound": "hbm",
                     "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4), "peak_source": peak_kind,
                     "alg_bytes_per_launch": int(alg_bytes),
                     "launch_ms": round(mean_solve_s * 1e3, 4), "cg_iterations": mean_iters,
                     "traffic": (traffic or {}).get("bytes_per_launch"),
                     "traffic_source": (traffic or {}).get("source")},
        "gpu_launches": int(launches),
        "clocks": clk,
        "modes": {"fp64": {"value": round(args.steps * world / (max_ms / 1e3), 3), "unit": "steps/s",
                           "solve_ms": round(mean_solve_s * 1e3, 4), "cg_iterations": mean_iters,
                           "dtype": "f64 (reference algorithms)"},
                  "fp32_refine": mixed},
    }
    return line


def bench_e2e(args, capi, rank):
    import numpy as np
    import torch

    def pinned(shape, dtype):
        tdt = {np.float64: torch.float64, np.int32: torch.int32}[dtype]
        return torch.empty(shape, dtype=tdt, pin_memory=True).numpy()

    run = make_run(capi, rank)
    s = run.sys
    for name in ("types", "pos", "vel", "mass", "charges", "pot_params"):
        a = getattr(s, name)
        p = pinned(a.shape, a.dtype.type)
        p[...] = a
        setattr(s, name, p)
    outs = {k: pinned((s.n_ions, 3), np.float64) for k in ("pos", "vel", "fcs_tot")}
    h2d = sum(getattr(s, k).nbytes for k in ("types", "pos", "vel", "mass", "charges", "pot_params"))
    d2h = sum(o.nbytes for o in outs.values()) + 4 + 4 + 8
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    run.initialize()
    for _ in range(args.steps):
        run.step()
        capi.get_pos(outs["pos"])
        capi.get_vel(outs["vel"])
        capi.get_fcs_tot(outs["fcs_tot"])
    seconds = time.perf_counter() - t0
    run.finalize()
    return {"seconds": seconds, "h2d": int(round(h2d / args.steps)), "d2h": int(d2h)}


def reference_lib():
    from oracle import loader
    return loader.REF_FAST_SO if os.path.exists(loader.REF_FAST_SO) else None


def cpu_baseline_sample(steps=2):
    """Reference C (shipped flags, OpenMP on all cores) on `steps` MD steps after init."""
    code = f"""
import json, os, sys, time
sys.path.insert(0, {ROOT!r})
from maze_poisson_b200.c_api import CAPI
import bench
run = bench.make_run(CAPI({reference_lib()!r}, extensions=False), 0)
run.initialize()
t0 = time.perf_counter()
for _ in range({steps}):
    run.step()
dt = time.perf_counter() - t0
run.finalize()
print(json.dumps({{"seconds": dt}}))
"""
    cores = os.cpu_count() or 1
    env = dict(os.environ, OMP_NUM_THREADS=str(cores))
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, env=env,
                       timeout=1800)
    dt = json.loads(r.stdout.strip().splitlines()[-1])["seconds"]
    return {"value": round(steps / dt, 4), "unit": "steps/s", "cores": cores, "kind": "reference",
            "sample": f"{steps} MD steps of nacl2000_128 after initialisation, reference C "
                      f"(-O3 --fast-math -mavx2, OpenMP {cores} threads)"}


def bench_reference(args):
    cores = os.cpu_count() or 1
    path = reference_lib()
    if path is None:
        print(json.dumps({"impl": "reference", "unavailable":
                          "reference build oracle/_ref/libmaze_poisson_ref_fast.so is missing"}))
        return
    os.environ["OMP_NUM_THREADS"] = str(cores)
    from maze_poisson_b200.c_api import CAPI
    capi = CAPI(path, extensions=False)
    run = make_run(capi, 0)
    run.initialize()
    for _ in range(args.warmup):
        run.step()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        run.step()
    dt = time.perf_counter() - t0
    run.finalize()
    v = round(args.steps / dt, 4)
    print(json.dumps({
        "metric": METRIC, "value": v, "unit": "steps/s", "n_gpus": 0, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(dt / args.steps * 1e3, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded NaCl lattice, jitter 0.1a, MB velocities)", "config": CONFIG,
        "impl": "reference",
        "cpu_baseline": {"value": v, "unit": "steps/s", "cores": cores, "kind": "reference",
                         "sample": f"{args.steps} full MD steps after {args.warmup} warm-up steps"},
        "e2e": {"value": v, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--fp64-only", action="store_true", help="skip the FP32+refine measurement")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))

    if args.impl == "reference":
        if rank == 0:
            bench_reference(args)
        return

    dist = None
    if world > 1:
        import datetime
        import torch.distributed as td
        td.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
        dist = td
    try:
        line = bench_b200(args, rank, world, dist)
        if rank == 0:
            if world == 1 and not args.no_cpu_baseline and reference_lib() is not None:
                line["cpu_baseline"] = cpu_baseline_sample()
            print(json.dumps(line), flush=True)
    finally:
        if dist is not None:
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
