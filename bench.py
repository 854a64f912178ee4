#!/usr/bin/env python
"""Benchmark of the MaZe_Poisson MD hot path on B200 (one JSON line on rank 0).

Workload (the mixed-precision configuration, N = 16000 / 256^3): 16000 Na+/Cl- ions at
1.379 g/cm^3 on a 20^3-cell lattice (Na at the corner, Cl at the body centre) with +-0.1a
jitter and 1200 K Maxwell-Boltzmann velocities; 256^3 grid, CIC spreading, field solve to
an absolute inf-norm residual of 1e-10, Tosi-Fumi forces with r_cut = L/2, velocity
Verlet, dt = 1 fs. Synthetic and seeded.

A step is one SolverMD.md_loop_iter (maze_poisson/solver.py:483-492): integrator part 1,
charge spreading, field solve, field + pair + total forces, integrator part 2.

Forms, each from the same initial state (`modes` in the JSON line):
  fp32_refine : the field solve is FP32 multigrid V-cycles inside FP64 iterative
                refinement (FP64 residual, correction, energies, positions) -- the headline
                `value`;
  fp64        : the reference's own algorithm (LCG: CG with implicit Jacobi) in FP64,
                within 1e-10 of the CPU oracle per step;
  fp64_multigrid_ref, fp64_maze_multigrid_ref : the reference's MULTIGRID and
                MAZE-MULTIGRID algorithms (2-level V-cycle, coarse CG) in FP64;
  fp64_mg     : the fair FP64 comparator of fp32_refine -- the same V(3,2) multigrid and
                refinement loop with every value in FP64;
  fft         : the reference's FFT Poisson method (a spectral discretisation, so it is
                timed beside the others but not counted among the FP64 comparators).
`speedup_fp32_refine_over_fp64` sets fp32_refine against the CG form;
`speedup_fp32_refine_over_best_fp64` against the fastest FP64 form that solves the same
7-point problem.
After the same steps the forces, energies and positions of fp32_refine and fp64_mg are
compared with fp64 (`errors_vs_fp64`). Then one MD step restarted from the FP64 state
(solver_set_field / solver_set_field_prev) is run by the reference's C on the host (the
cpu_baseline) and by each GPU form, and the GPU results are compared with the C's
(`errors_vs_reference_c`).

  value : steps/s of fp32_refine with the state resident on the GPU, each step run by
          solver_md_step(1) and timed with CUDA events on the library's stream; L2 (126 MB)
          is flushed by writing a 256 MB buffer on that stream before every timed step
          (outside the events). N GPUs run N independent replicas (weak scaling); the job's
          value is total steps / max-over-ranks time.
  e2e   : steps/s of a whole fp32_refine job through the reference's ctypes ABI from host
          buffers: solver_initialize_particles (H2D from pinned host memory), the two
          bootstrap steps, then K steps of the reference's per-call sequence, each followed
          by get_pos/get_vel/get_fcs_tot (D2H into pinned host memory); wall clock / K.
  roofline : the mixed field-solve kernel (one launch per step) against the measured HBM
          copy bandwidth, with algorithmic bytes per launch from mixed_solve_bytes().

`--impl reference` times the reference's own C library (built from its sources, shipped
Release flags, OpenMP on every host core) through its facade on the same workload, with
its fastest method here (MAZE-MULTIGRID) as the line's value and LCG beside it.
"""
import argparse
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

METRIC = "MD steps/s, FP32+refine field solve (FP64 plain beside it), N=16000 / 256^3"
WORKLOAD = dict(ncell=20, n_grid=256, density=1.379)
SOLVER = dict(method="LCG", precond="NONE", tol=1e-10, integrator="VERLET", thermostat=False, T=1200.0,
              gamma_per_ps=1.0, dt_fs=1.0)
CONFIG = {"workload": "nacl16000_256", "n_ions": 16000, "grid": 256, "density_g_cm3": 1.379,
          "method": "FP32 multigrid + FP64 refinement (fp32_refine); FP64 forms LCG, MULTIGRID, "
                    "MAZE-MULTIGRID and FP64 multigrid beside it; reference C: MAZE-MULTIGRID and LCG",
          "tol": 1e-10,
          "integrator": "VERLET", "dt_fs": 1.0, "T0_K": 1200,
          "l2": "flushed (256 MB write) before every timed step", "parallelism": "replicas"}
DATA = "synthetic (seeded NaCl 2-ion-cell lattice, jitter 0.1a, 1200 K MB velocities)"


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def load_traffic():
    """Per-launch DRAM bytes of the mixed solve kernel from a committed ncu summary, if any."""
    try:
        with open(os.path.join(ROOT, "profiles", "mixed_kernel_traffic.json")) as f:
            return json.load(f)
    except Exception:
        return None


def level_sizes(n):
    """Multigrid levels of the mixed solver: n, n/2, ... while the next size is even and >= 4."""
    sizes = [n]
    m = n
    while m % 2 == 0 and (m // 2) % 2 == 0 and m // 2 >= 4 and len(sizes) < 10:
        m //= 2
        sizes.append(m)
    return sizes


def fft_coarse_level(n):
    """The coarse level the mixed solver solves by FFT (n/2 when that is 32, 64 or 128 points
    per side), or None when its hierarchy ends at a level of at most 16 points per side."""
    m = n // 2
    return m if n % 2 == 0 and m in (32, 64, 128) else None


def mixed_solve_bytes(n, refinements, nu1=3, nu2=2, small_n=16, w0=None):
    """Algorithmic HBM bytes of one mixed solve (MD update, LCG form) that took
    `refinements` V(nu1, nu2)-cycles (the library's default V(3,2)), with 8 B per FP64 value,
    4 B per FP32 value of the coarser levels and w0 B per value of level 0's correction,
    rhs and residual (2: FP16, which the library takes at n = 256; else 4), per grid point:
      set-up          read q, phi_old; write y, rhs, phi                     40 B
      residual check  read X, q; write level-0 rhs, red e      16 + 1.5 w0 B, refinements + 1 times
      update          read X, e; write X                             16 + w0 B
      V-cycle, per point of each level swept by the whole grid, with the red-black split
      layout (a half-sweep reads the other colour, this colour's rhs and writes this
      colour: 3 x w x 1/2):
        2 nu1 - 1 + 2 nu2 half-sweeps                              1.5 w each
        red residual: read both colours of x, red rhs; write red r       2 w
        restriction (13 red taps): read red r; write coarse rhs, x     w / 2 + 2 w_c / 8
        prolongation into black points: read coarse x; read/write black  w_c / 8 + w
      (w the level's value size, w_c the next level's, 4 B)
      coarse level of m points per side solved by FFT (fft_coarse_level): read its rhs,
        write x (4 B each), the half spectrum m^2 (m/2 + 1) complex (8 B) written by the
        first pass, read and written by the second, read by the third:  8 m^3 + 32 m^2 (m/2 + 1)
    Otherwise levels of at most small_n^3 points are solved in shared memory or from a
    staged Green's function and move no HBM bytes."""
    if w0 is None:
        w0 = 2 if n == 256 else 4
    P = n ** 3

    def per_level(w):
        return (2 * nu1 - 1 + 2 * nu2) * 1.5 * w + 2 * w + (w / 2 + 1) + (0.5 + w)

    m = fft_coarse_level(n)
    if m is not None:
        vcycle = P * per_level(w0) + 8 * m ** 3 + 32 * m * m * (m // 2 + 1)
    else:
        grid_levels = [k for k in level_sizes(n) if k > small_n]
        vcycle = sum(k ** 3 * per_level(w0 if k == n else 4) for k in grid_levels)
    return P * 40 + (refinements + 1) * P * (16 + 1.5 * w0) + refinements * (vcycle + P * (16 + w0))


class ClockSampler:
    """SM clock and throttle reasons sampled every 10 ms during the timed region through
    NVML (the library nvidia-smi reads; read-only queries). The GPU is found by the CUDA
    device's UUID, so CUDA_VISIBLE_DEVICES remapping does not pick another GPU."""

    REASONS = (("hw_slowdown", "nvmlClocksEventReasonHwSlowdown"),
               ("hw_thermal_slowdown", "nvmlClocksEventReasonHwThermalSlowdown"),
               ("sw_thermal_slowdown", "nvmlClocksEventReasonSwThermalSlowdown"),
               ("sw_power_cap", "nvmlClocksEventReasonSwPowerCap"))

    def __init__(self, index, period_s=0.01):
        self.index = index
        self.period = period_s
        self.samples = []
        self.thread = None
        self.stop_ev = threading.Event()

    def start(self):
        try:
            import pynvml
            import torch
            pynvml.nvmlInit()
            uuid = str(torch.cuda.get_device_properties(self.index).uuid)
            if not uuid.startswith("GPU-"):
                uuid = "GPU-" + uuid
            self.nvml = pynvml
            self.handle = pynvml.nvmlDeviceGetHandleByUUID(uuid)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self.handle, pynvml.NVML_CLOCK_SM)
        except Exception as e:  # no NVML: report the absence instead of a number
            self.error = f"{type(e).__name__}: {e}"
            return
        self.thread = threading.Thread(target=self._loop, daemon=True)
        self.thread.start()

    def _loop(self):
        nv, h = self.nvml, self.handle
        masks = [(name, getattr(nv, attr)) for name, attr in self.REASONS]
        while True:
            sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
            r = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
            self.samples.append((sm, [name for name, m in masks if r & m]))
            if self.stop_ev.wait(self.period):
                return

    def stop(self):
        if self.thread is None:
            return {"error": getattr(self, "error", "sampler not started")}
        self.stop_ev.set()
        self.thread.join()
        try:
            self.nvml.nvmlShutdown()
        except Exception:
            pass
        reasons = sorted({n for _, rs in self.samples for n in rs})
        return {"sm_mhz": statistics.median(s for s, _ in self.samples), "sm_max_mhz": self.max_mhz,
                "reasons": reasons, "samples": len(self.samples), "source": "NVML, 10 ms"}


# mode -> (method, precision): the headline form first, then the FP64 forms
FORMS = {
    "fp32_refine": ("LCG", 1),
    "fp64": ("LCG", 0),
    "fp64_multigrid_ref": ("MULTIGRID", 0),
    "fp64_maze_multigrid_ref": ("MAZE-MULTIGRID", 0),
    "fp64_mg": ("LCG", 2),
    "fft": ("FFT", 0),
}
# forms that solve the same 7-point discretisation as fp32_refine (FFT solves the
# spectral one, so it is timed beside them but not counted as an FP64 comparator)
SAME_PROBLEM_FP64 = ("fp64", "fp64_multigrid_ref", "fp64_maze_multigrid_ref", "fp64_mg")
FORM_DTYPE = {
    "fp32_refine": "f32 multigrid bulk + f64 residual/refinement/energies/positions",
    "fp64": "f64 (the reference's LCG algorithm)",
    "fp64_multigrid_ref": "f64 (the reference's MULTIGRID algorithm)",
    "fp64_maze_multigrid_ref": "f64 (the reference's MAZE-MULTIGRID algorithm)",
    "fp64_mg": "f64 (the V(3,2) multigrid + refinement loop of fp32_refine, every value in FP64)",
    "fft": "f64 (the reference's FFT Poisson solve, continuous k^2; hand-written shared-memory FFT)",
}


def fft_solve_bytes(n):
    """Algorithmic HBM bytes of one FFT solve (five passes): r2c along k reads q (8 B per
    point) and writes the n x n x (n/2+1) complex spectrum (16 B per value); the three column
    passes (forward j; forward i, multiply, inverse i; inverse j) read and write it; c2r
    reads it and writes phi."""
    spec = n * n * (n // 2 + 1) * 16
    return 2 * 8 * n ** 3 + 8 * spec


def make_run(capi, rank, precision=0, method=None):
    from maze_poisson_b200.md import MDRun
    from maze_poisson_b200.systems import make_system
    system = make_system(seed=1000 + rank, T=SOLVER["T"], **WORKLOAD)
    kw = dict(SOLVER)
    if method is not None:
        kw["method"] = method
    return MDRun(capi, system, precision=precision, **kw)


def timed_steps(capi, stream, flush, steps):
    """Device time of `steps` MD steps (CUDA events on the library stream, L2 flushed
    before each), the solve times and the solver's return values."""
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


def run_form(args, capi, rank, local, precision, flush, dist, sample_clocks=False, method=None, keep_fields=False):
    """W warm-up + K timed steps of one form; returns timings and the final state."""
    import numpy as np
    import torch
    run = make_run(capi, rank, precision, method)
    run.initialize()
    stream = torch.cuda.ExternalStream(capi.mzb_get_stream(), device=local)
    for _ in range(args.warmup):
        capi.solver_md_step(1)
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(local) if sample_clocks else None
    if clocks:
        clocks.start()
    l0 = capi.mzb_kernel_launches()
    total_ms, solve_ms, iters = timed_steps(capi, stream, flush, args.steps)
    launches = capi.mzb_kernel_launches() - l0
    clk = clocks.stop() if clocks else None
    st = run.state(fields=False)
    g = WORKLOAD["n_grid"]
    q = np.empty((g, g, g), dtype=np.float64)
    phi = np.empty((g, g, g), dtype=np.float64)
    capi.get_q(q)
    capi.get_field(phi)
    st["u_elec"] = 0.5 * float(np.dot(q.ravel(), phi.ravel()))  # 1/2 sum_grid q phi, FP64
    del q, phi
    fields = None
    if keep_fields:
        fields = {}
        for name in ("field", "field_prev"):
            a = np.empty((g, g, g), dtype=np.float64)
            getattr(capi, "get_" + name)(a)
            fields[name] = a
    run.finalize()
    t = torch.tensor([total_ms], dtype=torch.float64, device=f"cuda:{local}")
    if dist is not None:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return {"ms": float(t.item()), "solve_ms": solve_ms, "iters": iters, "launches": launches,
            "clocks": clk, "state": st, "fields": fields}


def rms_rel(a, b):
    import numpy as np
    return float(np.sqrt(np.mean((a - b) ** 2)) / np.sqrt(np.mean(b ** 2)))


def bench_b200(args, rank, world, dist):
    import numpy as np
    import torch

    local = int(os.environ.get("LOCAL_RANK", "0"))
    os.environ["MZB_DEVICE"] = str(local)
    os.environ.setdefault("MZB_QUIET", "1")
    torch.cuda.set_device(local)
    from maze_poisson_b200.c_api import CAPI
    capi = CAPI()
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=f"cuda:{local}")

    forms = {}
    for name, (method, precision) in FORMS.items():
        forms[name] = run_form(args, capi, rank, local, precision, flush, dist, sample_clocks=name == "fp32_refine",
                               method=method, keep_fields=name == "fp64" and args.cpu_fields is not None)
    mix, f64 = forms["fp32_refine"], forms["fp64"]
    del flush

    # end to end through the reference ABI from pinned host buffers (fp32_refine)
    e2e = bench_e2e(args, capi, rank, precision=1)
    if dist is not None:
        et = torch.tensor([e2e["seconds"]], dtype=torch.float64, device=f"cuda:{local}")
        dist.all_reduce(et, op=dist.ReduceOp.MAX)
        e2e["seconds"] = float(et.item())

    def errors_vs(a, b):
        return {"fcs_tot_rms_rel": rms_rel(a["fcs_tot"], b["fcs_tot"]),
                "fcs_tot_max_rel": max_rel(a["fcs_tot"], b["fcs_tot"]),
                "fcs_elec_rms_rel": rms_rel(a["fcs_elec"], b["fcs_elec"]),
                "fcs_noel_rms_rel": rms_rel(a["fcs_noel"], b["fcs_noel"]),
                "pos_max_abs_bohr": float(np.abs(a["pos"] - b["pos"]).max()),
                "u_elec_rel": abs(a["u_elec"] - b["u_elec"]) / abs(b["u_elec"]),
                "potential_notelec_rel": abs(a["potential_notelec"] - b["potential_notelec"]) /
                abs(b["potential_notelec"]),
                "kinetic_rel": abs(a["kinetic"] - b["kinetic"]) / abs(b["kinetic"])}

    after = f"{args.warmup + args.steps} MD steps from the same initial state"
    errors = dict(errors_vs(mix["state"], f64["state"]), compared_after=after)
    errors_mg = dict(errors_vs(forms["fp64_mg"]["state"], f64["state"]), compared_after=after)

    # one MD step restarted from the FP64 state by each GPU form (compared with the
    # reference's C on the same step, cpu_baseline_sample)
    restarted = None
    if f64["fields"] is not None:
        start = {"pos": f64["state"]["pos"], "vel": f64["state"]["vel"], **f64["fields"]}
        restarted = {name: restarted_step(capi, rank, FORMS[name][1], FORMS[name][0], start)
                     for name in ("fp64", "fp32_refine", "fp64_mg")}
        for name in ("field", "field_prev"):
            np.save(os.path.join(args.cpu_fields, f"{name}.npy"), f64["fields"][name])
        np.save(os.path.join(args.cpu_fields, "pos.npy"), f64["state"]["pos"])
        np.save(os.path.join(args.cpu_fields, "vel.npy"), f64["state"]["vel"])
        f64["fields"] = None

    n = WORKLOAD["n_grid"]
    mean_solve_s = statistics.mean(mix["solve_ms"]) / 1e3
    mean_ref = statistics.mean(mix["iters"])
    alg_bytes = mixed_solve_bytes(n, mean_ref)
    peak, peak_kind = load_peaks()
    achieved = alg_bytes / mean_solve_s / 1e9
    traffic = load_traffic()

    def steps_s(ms):
        return round(args.steps * world / (ms / 1e3), 3)

    modes = {}
    for name, f in forms.items():
        method, precision = FORMS[name]
        m = {"value": steps_s(f["ms"]), "unit": "steps/s", "ms_per_step": round(f["ms"] / args.steps, 4),
             "solve_ms": round(statistics.mean(f["solve_ms"]), 4), "method": method, "precision": precision,
             "solver_result_mean": statistics.mean(f["iters"]), "gpu_launches": int(f["launches"]),
             "dtype": FORM_DTYPE[name]}
        modes[name] = m
    modes["fp32_refine"]["errors_vs_fp64"] = errors
    modes["fp64_mg"]["errors_vs_fp64"] = errors_mg
    best = min(SAME_PROBLEM_FP64, key=lambda k: forms[k]["ms"])
    fft_s = statistics.mean(forms["fft"]["solve_ms"]) / 1e3
    modes["fft"]["roofline"] = {"kernel": "FFT passes (k_pass_k_fwd, k_pass_cols x3, k_pass_k_inv)", "bound": "hbm",
                                "alg_bytes_per_solve": fft_solve_bytes(n),
                                "achieved": round(fft_solve_bytes(n) / fft_s / 1e9, 1), "peak": peak,
                                "unit": "GB/s", "frac": round(fft_solve_bytes(n) / fft_s / 1e9 / peak, 4)}
    modes["speedup_fp32_refine_over_fp64"] = round(f64["ms"] / mix["ms"], 3)
    modes["speedup_fp32_refine_over_best_fp64"] = round(forms[best]["ms"] / mix["ms"], 3)
    modes["best_fp64_form"] = best

    line = {
        "metric": METRIC,
        "value": steps_s(mix["ms"]),
        "unit": "steps/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(mix["ms"] / args.steps, 4),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": FORM_DTYPE["fp32_refine"],
        "data": DATA,
        "config": CONFIG,
        "e2e": {"value": round(args.steps * world / e2e["seconds"], 3), "unit": "steps/s",
                "h2d_bytes_per_step": e2e["h2d"], "d2h_bytes_per_step": e2e["d2h"]},
        "roofline": {"kernel": "mixed_kernel (FP32 multigrid + FP64 refinement field solve)", "bound": "hbm",
                     "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4), "peak_source": peak_kind,
                     "alg_bytes_per_launch": int(alg_bytes),
                     "launch_ms": round(mean_solve_s * 1e3, 4), "refinements": mean_ref,
                     "traffic": (traffic or {}).get("bytes_per_launch"),
                     "traffic_source": (traffic or {}).get("source")},
        "gpu_launches": int(mix["launches"]),
        "clocks": mix["clocks"],
        "modes": modes,
    }
    if traffic and traffic.get("bytes_per_launch"):
        line["roofline"]["frac_of_dram_traffic"] = round(traffic["bytes_per_launch"] / mean_solve_s / 1e9 / peak, 4)
    return line, restarted


def max_rel(a, b):
    import numpy as np
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


def restarted_step(capi, rank, precision, method, start):
    """One MD step of a GPU form restarted from `start` (MDRun.restart); its results."""
    import numpy as np
    run = make_run(capi, rank, precision, method)
    run.restart(start["pos"], start["vel"], start["field"], start["field_prev"])
    try:
        run.step()
        st = run.state(fields=False)
        g = WORKLOAD["n_grid"]
        q, phi = np.empty((g, g, g)), np.empty((g, g, g))
        capi.get_q(q)
        capi.get_field(phi)
        st["u_elec"] = 0.5 * float(np.dot(q.ravel(), phi.ravel()))
    finally:
        run.finalize()
    return st


def bench_e2e(args, capi, rank, precision):
    import numpy as np
    import torch

    def pinned(shape, dtype):
        tdt = {np.float64: torch.float64, np.int32: torch.int32}[dtype]
        return torch.empty(shape, dtype=tdt, pin_memory=True).numpy()

    run = make_run(capi, rank, precision)
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


CPU_SAMPLE = r"""
import json, os, sys, time
import numpy as np
sys.path.insert(0, {root!r})
from maze_poisson_b200.c_api import CAPI
import bench
capi = CAPI({lib!r}, extensions=False)
d = {fields!r}
start = {{k: np.load(os.path.join(d, k + ".npy")) for k in ("pos", "vel", "field", "field_prev")}}
out = {{}}
for method, steps in {plan!r}:
    run = {make_run}
    run.restart(start["pos"], start["vel"], start["field"], start["field_prev"])
    times = []
    for _ in range(steps):
        t0 = time.perf_counter()
        run.step()
        times.append(time.perf_counter() - t0)
    out[method] = {{"seconds": times[-1], "iters": run.n_iters}}
    if {dump!r} and method == {plan!r}[0][0]:
        st = run.state(fields=False)
        g = run.sys.n_grid
        q, phi = np.empty((g, g, g)), np.empty((g, g, g))
        capi.get_q(q)
        capi.get_field(phi)
        st["u_elec"] = 0.5 * float(np.dot(q.ravel(), phi.ravel()))
        np.savez(os.path.join(d, "ref_step.npz"), **{{k: np.asarray(v) for k, v in st.items() if v is not None}})
    run.finalize()
print(json.dumps(out))
"""


def cpu_baseline_sample(fields_dir):
    """The reference's C (shipped flags, OpenMP on all cores) restarted
    (solver_set_field / solver_set_field_prev) from the FP64 GPU form's state after its
    timed steps, as the reference's restart path does: one LCG step (its results are kept
    for errors_vs_reference_c) and two MAZE-MULTIGRID steps, of which the second is timed
    (the first starts the MaZe auxiliary field from zero). The value is the faster method."""
    import numpy as np
    cores = os.cpu_count() or 1
    plan = [("LCG", 1), ("MAZE-MULTIGRID", 2)]
    code = CPU_SAMPLE.format(root=ROOT, lib=reference_lib(), fields=fields_dir, plan=plan, dump=True,
                             make_run="bench.make_run(capi, 0, 0, method)")
    env = dict(os.environ, OMP_NUM_THREADS=str(cores))
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, env=env, timeout=1800)
    if r.returncode != 0:
        return {"unavailable": (r.stderr.strip().splitlines() or ["cpu sample failed"])[-1][:200]}, None
    out = json.loads(r.stdout.strip().splitlines()[-1])
    best = min(out, key=lambda m: out[m]["seconds"])
    per = {m: {"value": round(1 / v["seconds"], 4), "unit": "steps/s", "solver_result": v["iters"]}
           for m, v in out.items()}
    ref = dict(np.load(os.path.join(fields_dir, "ref_step.npz")))
    return ({"value": per[best]["value"], "unit": "steps/s", "cores": cores, "kind": "reference",
             "method": best, "methods": per,
             "sample": f"1 MD step of nacl16000_256 restarted from the FP64 GPU state (LCG; for "
                       f"MAZE-MULTIGRID the second of 2 steps), tol 1e-10; reference C (-O3 --fast-math "
                       f"-mavx2, OpenMP {cores} threads); value = the faster method ({best})"}, ref)


# Poisson-Boltzmann workload (--workload pb_solute32_128): a 32-ion Na+/Cl- solute (a
# cluster of radius 10 A, ions >= 2.7 A apart) at the centre of a 40 A box of implicit
# water (eps_s 78.4, eps_int 1, 0.15 M ionic strength, shell half-width 1 bohr, non-polar
# forces on), 128^3 grid (h = 0.3125 A), Tosi-Fumi pairs, Verlet at 300 K, dt 1 fs.
PB_WORKLOAD = dict(n_ions=32, n_grid=128, box_ang=40.0, cluster_ang=10.0, seed=11)
PB_SOLVER = dict(tol=1e-10, integrator="VERLET", T=300.0, eps_s=78.4, eps_int=1.0, dt_fs=1.0)


def make_pb_run(capi, method):
    from maze_poisson_b200.md import MDRun
    from maze_poisson_b200.systems import make_pb_system, pb_settings
    w = PB_WORKLOAD
    s = make_pb_system(w["n_ions"], w["n_grid"], w["box_ang"], T=PB_SOLVER["T"], seed=w["seed"],
                       cluster_ang=w["cluster_ang"])
    return MDRun(capi, s, method=method, pb=pb_settings(s, eps_s=PB_SOLVER["eps_s"]), **PB_SOLVER)


def pb_cg_bytes(n, iterations):
    """Algorithmic bytes of one PB CG solve: per iteration 8 values of the Poisson CG
    (x, r, p read + write; Ap write + read) plus the 4 operator coefficients (ex, ey, ez,
    dg) read once, 8 bytes each per point; set-up: b, x0, the 4 coefficients read, r and x
    written."""
    P = n ** 3
    return P * 8 * (12 * iterations + 8)


def bench_pb(args):
    """One JSON line: GPU steps/s of the PB workload (FP64, the reference's PB algorithms)
    with per-phase device times, the solve kernel's roofline (CG methods) and the
    reference's C on the host cores for one step restarted from the GPU state."""
    import numpy as np
    import torch
    from maze_poisson_b200.c_api import CAPI
    os.environ.setdefault("MZB_QUIET", "1")
    torch.cuda.set_device(0)
    capi = CAPI()
    run = make_pb_run(capi, args.method)
    run.initialize()
    stream = torch.cuda.ExternalStream(capi.mzb_get_stream(), device=0)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda:0")
    for _ in range(args.warmup):
        capi.solver_md_step(1)
    torch.cuda.synchronize()
    clocks = ClockSampler(0)
    clocks.start()
    l0 = capi.mzb_kernel_launches()
    total_ms, solve_ms, iters = timed_steps(capi, stream, flush, args.steps)
    launches = capi.mzb_kernel_launches() - l0
    clk = clocks.stop()
    # phase split: the same calls as solver_md_step, each bracketed by events
    names = ("integrator_part_1", "solver_update_charges", "solver_update_eps_k2", "solver_update_field",
             "solver_compute_forces_elec", "solver_compute_forces_noel", "solver_compute_forces_pb",
             "solver_compute_forces_tot", "integrator_part_2")
    phase = {k: 0.0 for k in names}
    for _ in range(args.steps):
        for k in names:
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            with torch.cuda.stream(stream):
                flush.fill_(1.0)
                e0.record(stream)
            getattr(capi, k)()
            with torch.cuda.stream(stream):
                e1.record(stream)
            torch.cuda.synchronize()
            phase[k] += e0.elapsed_time(e1)
    want_cpu = not args.no_cpu_baseline and reference_lib() is not None
    cpu = None
    if want_cpu:
        with tempfile.TemporaryDirectory() as d:
            g = run.sys.n_grid
            for name in ("field", "field_prev"):
                a = np.empty((g, g, g))
                getattr(capi, "get_" + name)(a)
                np.save(os.path.join(d, f"{name}.npy"), a)
            st = run.state(fields=False)
            np.save(os.path.join(d, "pos.npy"), st["pos"])
            np.save(os.path.join(d, "vel.npy"), st["vel"])
            cores = os.cpu_count() or 1
            code = CPU_SAMPLE.format(root=ROOT, lib=reference_lib(), fields=d, plan=[(args.method, 1)], dump=False,
                                     make_run="bench.make_pb_run(capi, method)")
            env = dict(os.environ, OMP_NUM_THREADS=str(cores))
            r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, env=env,
                               timeout=1800)
            if r.returncode == 0:
                out = json.loads(r.stdout.strip().splitlines()[-1])[args.method]
                cpu = {"value": round(1 / out["seconds"], 5), "unit": "steps/s", "cores": cores,
                       "kind": "reference",
                       "sample": f"1 MD step of pb_solute32_128 ({args.method}, tol 1e-10, solver returned "
                                 f"{out['iters']}), restarted from the GPU state; reference C (-O3 --fast-math "
                                 f"-mavx2, OpenMP {cores} threads)"}
            else:
                cpu = {"unavailable": (r.stderr.strip().splitlines() or ["cpu sample failed"])[-1][:200]}
    run.finalize()
    peak, peak_kind = load_peaks()
    n = PB_WORKLOAD["n_grid"]
    mean_solve = statistics.mean(solve_ms)
    line = {
        "metric": f"PB MD steps/s (FP64, {args.method}), 32-ion solute in implicit water, 128^3",
        "value": round(args.steps / (total_ms / 1e3), 3), "unit": "steps/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(total_ms / args.steps, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded 32-ion NaCl cluster, 300 K MB velocities)",
        "config": {"workload": "pb_solute32_128", **PB_WORKLOAD, **PB_SOLVER, "method": args.method,
                   "l2": "flushed (256 MB write) before every timed step"},
        "phases_ms": {k: round(v / args.steps, 4) for k, v in phase.items()},
        "solve_ms": round(mean_solve, 4), "solver_result": iters[-1],
        "gpu_launches": int(launches), "clocks": clk,
    }
    if args.method in ("LCG", "MAZE-LCG") and iters[-1] > 0:
        it = statistics.mean(iters) + 1
        achieved = pb_cg_bytes(n, it) / (mean_solve / 1e3) / 1e9
        line["roofline"] = {"kernel": "engine_kernel (PB CG solve)", "bound": "hbm", "achieved": round(achieved, 1),
                            "peak": peak, "unit": "GB/s", "frac": round(achieved / peak, 4),
                            "peak_source": peak_kind, "alg_bytes_per_launch": int(pb_cg_bytes(n, it)),
                            "cg_iterations": it, "traffic": None}
    if cpu is not None:
        line["cpu_baseline"] = cpu
    print(json.dumps(line), flush=True)


# Batched workload (--workload batch64): 64 resident +-1 melts, N log-uniform in
# [128, 4000] (even), density from {1.329, 1.379} g/cm^3, grid from {32, 64, 96, 128}^3
# closest to 0.3 A spacing, FP32+refine to 1e-10, OVRVO at 1200 K with 1 ps^-1 friction,
# dt 1 fs, 300 steps, all replicas advanced by mzb_batch_step (a CUDA graph per MD step,
# one cooperative launch for all field solves) after mzb_batch_autotune.
BATCH = dict(count=64, seed=2026, steps=300)
BATCH_SOLVER = dict(method="LCG", tol=1e-10, integrator="OVRVO", thermostat=True, T=1200.0, gamma_per_ps=1.0,
                    dt_fs=1.0)


def make_replica(capi, spec, precision=1, method=None):
    from maze_poisson_b200.md import MDRun
    from maze_poisson_b200.systems import make_melt
    n, g, rho, seed = spec
    kw = dict(BATCH_SOLVER)
    if method is not None:
        kw["method"] = method
    return MDRun(capi, make_melt(n, g, density=rho, seed=seed), precision=precision, **kw)


def bench_batch(args):
    """One JSON line: replica-steps/s of the 64 replicas advanced together, beside the same
    replicas stepped one at a time alone on the GPU (each 3 warm-up + 10 timed steps,
    CUDA events, scaled to the batch's step count) and the reference's C on a sample of
    them on the host cores."""
    import numpy as np
    import torch
    from maze_poisson_b200.c_api import CAPI
    from maze_poisson_b200.systems import replica_set
    os.environ.setdefault("MZB_QUIET", "1")
    torch.cuda.set_device(0)
    capi = CAPI()
    reps = replica_set(BATCH["count"], BATCH["seed"])
    steps = args.batch_steps
    # alone: one replica resident at a time
    alone_ms = []
    for spec in reps:
        h = capi.mzb_system_create()
        run = make_replica(capi, spec)
        run.initialize()
        for _ in range(3):
            capi.solver_md_step(1)
        stream = torch.cuda.ExternalStream(capi.mzb_get_stream(), device=0)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            e0.record(stream)
        capi.solver_md_step(10)
        with torch.cuda.stream(stream):
            e1.record(stream)
        torch.cuda.synchronize()
        alone_ms.append(e0.elapsed_time(e1) / 10)
        run.finalize()
        capi.mzb_system_destroy(h)
    # together
    handles, runs = [], []
    for spec in reps:
        handles.append(capi.mzb_system_create())
        run = make_replica(capi, spec)
        run.initialize()
        runs.append(run)
    hs = np.array(handles, dtype=np.int32)
    tuned = np.zeros(4)
    t0 = time.perf_counter()
    capi.mzb_batch_autotune(hs, len(hs), tuned)
    tune_s = time.perf_counter() - t0
    capi.mzb_batch_step(hs, len(hs), args.warmup)
    torch.cuda.synchronize()
    clocks = ClockSampler(0)
    clocks.start()
    l0 = capi.mzb_kernel_launches()
    t0 = time.perf_counter()
    rc = capi.mzb_batch_step(hs, len(hs), steps)
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    launches = capi.mzb_kernel_launches() - l0
    clk = clocks.stop()
    for h in handles:
        capi.mzb_system_select(h)
        capi.solver_finalize()
        capi.mzb_system_destroy(h)
    value = len(reps) * steps / wall
    alone_s = sum(alone_ms) / 1e3 * steps
    points = [g ** 3 for _, g, _, _ in reps]
    line = {
        "metric": "replica MD steps/s, 64 replicas advanced together (FP32+refine, OVRVO)",
        "value": round(value, 2), "unit": "replica-steps/s", "n_gpus": 1, "steps": steps, "warmup": args.warmup,
        "ms_per_step": round(wall / steps * 1e3, 4), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32 multigrid bulk + f64 residual/refinement/energies/positions",
        "data": f"synthetic (seeded: replica_set(count={BATCH['count']}, seed={BATCH['seed']}), make_melt)",
        "config": {"workload": "batch64", "replicas": len(reps), "ions_total": int(sum(n for n, _, _, _ in reps)),
                   "grids": {str(g): sum(1 for _, x, _, _ in reps if x == g) for g in (32, 64, 96, 128)},
                   "grid_points_total": int(sum(points)), **BATCH_SOLVER, "tol": 1e-10,
                   "l2": "not flushed (a batched step moves several GB)"},
        "batch_rc": rc, "autotune": {"alpha": tuned[0], "ctas": tuned[1], "solve_ms": tuned[2],
                                      "forces_ms": tuned[3], "seconds": round(tune_s, 3)},
        "alone_gpu": {"value": round(len(reps) * steps / alone_s, 2), "unit": "replica-steps/s",
                      "sum_ms_per_step": round(sum(alone_ms), 4),
                      "sample": "each replica alone on the whole GPU, 10 timed steps after 3 warm-up steps"},
        "speedup_over_alone": round(alone_s / wall, 3),
        "gpu_launches": int(launches), "clocks": clk,
    }
    if not args.no_cpu_baseline and reference_lib() is not None:
        line["cpu_baseline"] = batch_cpu_sample(reps)
    print(json.dumps(line), flush=True)


BATCH_CPU = r"""
import json, sys, time
sys.path.insert(0, {root!r})
from maze_poisson_b200.c_api import CAPI
import bench
capi = CAPI({lib!r}, extensions=False)
out = []
for spec in {sample!r}:
    run = bench.make_replica(capi, tuple(spec), 0, "MAZE-MULTIGRID")
    run.initialize()
    run.step()
    t0 = time.perf_counter()
    run.step()
    out.append(time.perf_counter() - t0)
    run.finalize()
print(json.dumps(out))
"""


def batch_cpu_sample(reps):
    """The reference's C (MAZE-MULTIGRID, its fastest method; OpenMP on every host core)
    on one replica of each grid size in the set (the median N of that size), one timed step
    after the bootstrap and a warm-up step; the sum over all replicas is estimated as
    each size's sample time times the number of replicas of that size."""
    cores = os.cpu_count() or 1
    by_grid = {}
    for spec in reps:
        by_grid.setdefault(spec[1], []).append(spec)
    sample = []
    for g, specs in sorted(by_grid.items()):
        specs = sorted(specs)
        sample.append(specs[len(specs) // 2])
    code = BATCH_CPU.format(root=ROOT, lib=reference_lib(), sample=[list(x) for x in sample])
    env = dict(os.environ, OMP_NUM_THREADS=str(cores))
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, env=env, timeout=1800)
    if r.returncode != 0:
        return {"unavailable": (r.stderr.strip().splitlines() or ["cpu sample failed"])[-1][:200]}
    times = json.loads(r.stdout.strip().splitlines()[-1])
    est = sum(t * len(by_grid[spec[1]]) for t, spec in zip(times, sample))
    return {"value": round(len(reps) / est, 4), "unit": "replica-steps/s", "cores": cores, "kind": "reference",
            "sample": f"reference C (MAZE-MULTIGRID, OpenMP {cores} threads), one step per grid size "
                      f"({', '.join(f'N={n} {g}^3: {t:.3f} s' for (n, g, _, _), t in zip(sample, times))}); "
                      f"all replicas one after another estimated as size sample x count = {est:.2f} s per step"}


def bench_reference(args):
    """The reference's C on the host cores through its facade, with its own bootstrap, on
    its two methods for this workload: MAZE-MULTIGRID (its fastest here; the line's value)
    and LCG (beside it). Bounded sample: a 256^3 step takes seconds to tens of seconds on
    the host cores, so per method the timed steps are capped at 2 and the warm-up at 1
    (the two bootstrap steps run before both)."""
    cores = os.cpu_count() or 1
    path = reference_lib()
    if path is None:
        print(json.dumps({"impl": "reference", "unavailable":
                          "reference build oracle/_ref/libmaze_poisson_ref_fast.so is missing"}))
        return
    os.environ["OMP_NUM_THREADS"] = str(cores)
    from maze_poisson_b200.c_api import CAPI
    capi = CAPI(path, extensions=False)
    steps = max(1, min(args.steps, 2))
    warm = min(args.warmup, 1)
    per = {}
    for method in ("MAZE-MULTIGRID", "LCG"):
        run = make_run(capi, 0, 0, method)
        run.initialize()
        for _ in range(warm):
            run.step()
        t0 = time.perf_counter()
        for _ in range(steps):
            run.step()
        dt = time.perf_counter() - t0
        run.finalize()
        per[method] = {"value": round(steps / dt, 4), "unit": "steps/s", "ms_per_step": round(dt / steps * 1e3, 3),
                       "solver_result_last": run.n_iters}
    v = per["MAZE-MULTIGRID"]["value"]
    sample = (f"{steps} MD steps per method after the 2 bootstrap steps and {warm} warm-up step (steps capped at 2 "
              f"and warm-up at 1 to bound the run), tol 1e-10; value = MAZE-MULTIGRID, the reference's fastest "
              f"method here; LCG in modes")
    print(json.dumps({
        "metric": METRIC, "value": v, "unit": "steps/s", "n_gpus": 0, "steps": steps,
        "warmup": warm, "ms_per_step": per["MAZE-MULTIGRID"]["ms_per_step"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": DATA, "config": CONFIG, "impl": "reference", "modes": per,
        "cpu_baseline": {"value": v, "unit": "steps/s", "cores": cores, "kind": "reference", "sample": sample},
        "e2e": {"value": v, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


def errors_vs_reference_c(restarted, ref):
    """Each GPU form's restarted step against the reference C's LCG step from the same
    state: RMS and max-norm relative force errors, positions, energies."""
    import numpy as np
    out = {"compared": "1 MD step restarted from the same FP64 state; reference C LCG, tol 1e-10"}
    for name, st in restarted.items():
        out[name] = {"fcs_tot_rms_rel": rms_rel(st["fcs_tot"], ref["fcs_tot"]),
                     "fcs_tot_max_rel": max_rel(st["fcs_tot"], ref["fcs_tot"]),
                     "fcs_elec_rms_rel": rms_rel(st["fcs_elec"], ref["fcs_elec"]),
                     "fcs_noel_rms_rel": rms_rel(st["fcs_noel"], ref["fcs_noel"]),
                     "pos_max_abs_bohr": float(np.abs(st["pos"] - ref["pos"]).max()),
                     "vel_max_rel": max_rel(st["vel"], ref["vel"]),
                     "u_elec_rel": abs(st["u_elec"] - float(ref["u_elec"])) / abs(float(ref["u_elec"])),
                     "potential_notelec_rel": abs(st["potential_notelec"] - float(ref["potential_notelec"])) /
                     abs(float(ref["potential_notelec"])),
                     "kinetic_rel": abs(st["kinetic"] - float(ref["kinetic"])) / abs(float(ref["kinetic"]))}
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", choices=["nacl16000_256", "pb_solute32_128", "batch64"], default="nacl16000_256",
                    help="pb_solute32_128: the Poisson-Boltzmann workload; batch64: the batched form "
                         "(one GPU each, their own JSON line)")
    ap.add_argument("--batch-steps", type=int, default=BATCH["steps"], help="timed batched steps of batch64")
    ap.add_argument("--method", default="MAZE-LCG", help="field method of the PB workload")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.workload == "pb_solute32_128":
        bench_pb(args)
        return
    if args.workload == "batch64":
        bench_batch(args)
        return
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))

    if args.impl == "reference":
        if rank == 0:
            bench_reference(args)
        return

    want_cpu = rank == 0 and world == 1 and not args.no_cpu_baseline and reference_lib() is not None
    tmp = tempfile.TemporaryDirectory() if want_cpu else None
    args.cpu_fields = tmp.name if tmp else None
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as td
        td.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
        dist = td
    try:
        line, restarted = bench_b200(args, rank, world, dist)
        if want_cpu:
            line["cpu_baseline"], ref = cpu_baseline_sample(args.cpu_fields)
            if ref is not None and restarted is not None:
                line["modes"]["errors_vs_reference_c"] = errors_vs_reference_c(restarted, ref)
        if rank == 0:
            print(json.dumps(line), flush=True)
    finally:
        if dist is not None:
            dist.destroy_process_group()
        if tmp is not None:
            tmp.cleanup()


if __name__ == "__main__":
    main()
