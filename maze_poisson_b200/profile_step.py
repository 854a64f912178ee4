"""Run a few MD steps of a named workload through the C ABI -- the command the committed
ncu summaries (profiles/) profile.

    python -m maze_poisson_b200.profile_step --workload nacl2000_128 --method LCG --steps 1

Launch order of the field-solver kernels: two solves from zero (the two bootstrap steps of
SolverMD.initialize_md) then one warm-started solve per step.
"""
import argparse
import os

from .c_api import CAPI
from .md import MDRun
from .systems import WORKLOADS, make_system


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="nacl2000_128", choices=sorted(WORKLOADS) + ["batch64"],
                    help="batch64: the 64 replicas of the batched configuration, --steps batched steps "
                         "after autotuning and 8 untimed ones, bracketed by cuProfilerStart/Stop")
    ap.add_argument("--method", default="LCG")
    ap.add_argument("--precond", default="NONE")
    ap.add_argument("--tol", type=float, default=1e-8)
    ap.add_argument("--integrator", default="OVRVO")
    ap.add_argument("--steps", type=int, default=1)
    ap.add_argument("--precision", type=int, default=0, help="0 FP64, 1 FP32 multigrid + FP64 refinement")
    ap.add_argument("--outputs", type=int, default=0,
                    help="take the reference's per-stride outputs every N steps (0: none), both ways")
    ap.add_argument("--restart-every", action="store_true",
                    help="with --outputs: the restart outputs (both fields) at every output step")
    ap.add_argument("--no-write", action="store_true", help="with --outputs: transfer only, write no file")
    args = ap.parse_args()
    os.environ.setdefault("MZB_QUIET", "1")
    if args.workload == "batch64":
        return batch_steps(args.steps)
    run = MDRun(CAPI(), make_system(seed=1, **WORKLOADS[args.workload]), method=args.method,
                precond=args.precond, tol=args.tol, integrator=args.integrator,
                thermostat=args.integrator.upper() == "OVRVO", precision=args.precision)
    capi = run.capi
    run.initialize()
    if args.outputs:
        import tempfile
        import time
        from .output import Outputs
        for mode in (False, True, False, True):
            with tempfile.TemporaryDirectory() as d:
                out = Outputs(capi, d, ["Na", "Cl"], run.sys.n_grid, stride=args.outputs,
                              use_snapshots=mode, write=not args.no_write).bind(run.sys.n_ions)
                t0 = time.perf_counter()
                for k in range(args.steps):
                    run.step()
                    if args.restart_every and k % args.outputs == 0:
                        out.restart_step = k
                    out.output(k, run.potential_notelec)
                out.close()
                dt = (time.perf_counter() - t0) / args.steps
            what = "per-stride + restart" if args.restart_every else "per-stride"
            print(f"{what} outputs every {args.outputs} steps via {'snapshots' if mode else 'getters'}"
                  f"{' (no files)' if args.no_write else ''}: {dt * 1e3:.3f} ms per step")
    else:
        for k in range(args.steps):
            it = run.step()
            print(f"step {k}: solve {capi.mzb_last_solve_ms():.4f} ms, solver returned {it}")
    run.finalize()
    print("ok")


def batch_steps(steps):
    """The batched configuration (systems.replica_set(64, 2026): +-1 melts of N log-uniform in
    128-4000 on 64^3-128^3 grids, FP32+refine to 1e-10, OVRVO at 1200 K, 1 ps^-1, 1 fs):
    autotune, 8 untimed batched steps, then `steps` batched steps between
    cuProfilerStart and cuProfilerStop (for `ncu --profile-from-start off`)."""
    import ctypes

    import numpy as np

    from .systems import make_melt, replica_set
    capi = CAPI()
    handles = []
    for n, g, rho, seed in replica_set(64, 2026):
        handles.append(capi.mzb_system_create())
        MDRun(capi, make_melt(n, g, density=rho, seed=seed), method="LCG", tol=1e-10, integrator="OVRVO",
              thermostat=True, T=1200.0, gamma_per_ps=1.0, dt_fs=1.0, precision=1).initialize()
    hs = np.array(handles, dtype=np.int32)
    tuned = np.zeros(4)
    capi.mzb_batch_autotune(hs, len(hs), tuned)
    capi.mzb_batch_step(hs, len(hs), 8)
    cuda = ctypes.CDLL("libcuda.so.1")  # the driver's profiler switches act on this thread's context
    cuda.cuCtxSynchronize()
    cuda.cuProfilerStart()
    rc = capi.mzb_batch_step(hs, len(hs), steps)
    cuda.cuCtxSynchronize()
    cuda.cuProfilerStop()
    for h in handles:
        capi.mzb_system_select(int(h))
        capi.solver_finalize()
        capi.mzb_system_destroy(int(h))
    print(f"batch64: {steps} batched steps profiled, solver returned {rc}; tuned {tuned.tolist()}")


if __name__ == "__main__":
    main()
