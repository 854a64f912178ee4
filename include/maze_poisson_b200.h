/*
 * Extensions of the B200 build of libmaze_poisson.so. None of these has a counterpart
 * in the reference's ctypes binding; they serve parity tests (kernel-level entry points
 * on plain host arrays) and callers that want several MD steps per call.
 *
 * Grid arrays are plain n^3 C-contiguous doubles, idx = (i*n + j)*n + k, periodic in all
 * axes (the reference's (n+2)-plane halo layout is not used). Every entry point needs
 * solver_initialize() first; the kernel-level ones allocate and free device work
 * buffers per call.
 */
#ifndef MAZE_POISSON_B200_H
#define MAZE_POISSON_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* n_steps x SolverMD.md_loop_iter (maze_poisson/solver.py:483-492) with electrostatic
   and non-electrostatic forces; cf. the reference's commented-out solver_md_loop_iter /
   solver_run_n_steps (library/src/solver_md.c:202-228). Returns the last
   solver_update_field value. */
int solver_md_step(int n_steps);

/* kernel-level entry points (reference semantics on plain n^3 arrays) */
void mzb_laplace(const double *u, double *out, int n);                     /* laplace.c:24-75 */
int mzb_conj_grad(const double *b, const double *x0, double *x, double tol, int n,
                  int precond);  /* plcg.c:28-90 (precond 0), plcg.c:104-166 (1 JACOBI, 2 MG, 3 SSOR, 4 BLOCKJACOBI) */
void mzb_ssor_apply(const double *u, double *out, int n);                  /* precond_ssor.c:1240-1252 */
void mzb_blockjacobi_apply(const double *u, double *out, int n);    /* precond_blockjacobi.c:173-206; n % 10 == 0 */
void mzb_smooth_rbgs(const double *rhs, double *x, int n, int iters);      /* multigrid.c:636-729 */
void mzb_restrict27(const double *fine, double *coarse, int n);            /* multigrid.c:523-594 */
void mzb_prolong_trilinear(const double *coarse, double *fine, int nc);    /* multigrid.c:393-463 */
int mzb_cg_coarse(const double *b, double *x, int n, int maxit, double rtol); /* multigrid.c:13-96 */
void mzb_mg_apply(const double *rhs, double *x, int n, int sm);            /* multigrid.c:99-168 */
void mzb_fft_poisson(const double *q, double *phi, int n, double L, double h); /* fftw_wrap.c:166-189 */

/* Poisson-Boltzmann kernel-level entry points; ex/ey/ez/k2 are n^3 arrays of each point's
   +x/+y/+z face dielectric coefficients and screening term (grid_general.c:138-301) */
void mzb_laplace_pb(const double *u, double *out, const double *ex, const double *ey,
                    const double *ez, const double *k2, int n);                 /* laplace.c:77-145 */
int mzb_conj_grad_pb(const double *b, const double *x0, double *x, double tol, int n,
                     const double *ex, const double *ey, const double *ez,
                     const double *k2);                                          /* plcg.c:169-238 */
void mzb_smooth_pb(const double *rhs, double *x, int n, int iters, const double *ex,
                   const double *ey, const double *ez, const double *k2);   /* multigrid_pb.c:544-640 */
void mzb_mg_pb_apply(const double *rhs, double *x, int n, int sm, const double *ex,
                     const double *ey, const double *ez, const double *k2); /* multigrid_pb.c:270-328 */
void mzb_restrict_pb(const double *ex, const double *ey, const double *ez, const double *k2,
                     double *cex, double *cey, double *cez, double *ck2, int n); /* multigrid_pb.c:330-527 */
/* the PB coefficients of the current grid after solver_update_eps_k2 (no reference getter) */
void mzb_get_pb_grids(double *ex, double *ey, double *ez, double *k2);

/* precision of the field solve: 0 = the reference's FP64 algorithms (default), 1 = FP32
   multigrid V-cycles with FP64 iterative refinement until the FP64 residual meets the
   grid's tol (or tol_override when > 0), 2 = the same multigrid and refinement loop with
   every value in FP64 (the FP64 multigrid form, the fair FP64 comparator of mode 1). Also
   selected by MZB_PRECISION=mixed / fp64mg at solver_initialize_grid. FFT grids and grids
   that cannot be halved twice stay on the reference's algorithms. No counterpart in the
   reference. */
void mzb_set_precision(int mode, double tol_override);
int mzb_get_precision(void);      /* precision in effect for the current grid */

/* coarse-level plan of the current grid's multigrid forms (precision 1 and 2): 0 = levels
   down to the first of at most 16 points per side, solved by its Green's function; 1 or 2 =
   the first level from level 1 or 2 on with 32, 64 or 128 points per side is solved by FFT;
   -1 = default (1). Returns -1 for an unknown plan. No counterpart in the reference. */
int mzb_set_mixed_plan(int plan);
int mzb_get_mixed_plan(void);     /* the level solved by FFT (1, 2) or 0 when none is */

/* red-black Gauss-Seidel sweeps before (nu1) and after (nu2) the coarse correction in the
   V-cycle of the current grid's multigrid forms (precision 1 and 2); 1 .. 16 each, default
   V(3,2); returns -1 outside that range. No counterpart in the reference (its multigrid,
   library/src/multigrid.c:111-124, takes 3 sweeps on 2 levels). */
int mzb_set_mixed_sweeps(int nu1, int nu2);
void mzb_get_mixed_sweeps(int *nu1, int *nu2);

/* state accessors of the current system */
void mzb_get_cic_neighbors(int64_t *out);  /* (n_p,8,3) CIC corners, particles.c:297-346 */
void mzb_set_cell_grid(int nc);            /* linked cells per side for the pair forces */
int mzb_get_cells(int32_t *start, int32_t *ions); /* CSR linked cells; returns nc */
void mzb_philox_normals(uint64_t call, double *out); /* O-block draws of call `call` (n_p,3) */
void mzb_set_seed(uint64_t seed);          /* O-block Philox key */
uint64_t mzb_get_ocalls(void);             /* O-blocks applied so far */

/* CG solve that allocates no device memory, for callers that cannot call cudaMalloc
   (a host framework that owns all device allocations, a loop that must not take an
   allocation's implicit synchronisation). No counterpart in the reference. b, x0, x are
   caller-owned buffers of n^3 doubles on the current device, 2 <= n <= 64; the work arrays
   live in a static ~8.4 MB device array that every GPU loading this library holds until
   exit and that all calls share (overlapping calls race). The first call per device looks
   up that array's address. The call is synchronous (it waits for the solve and reads the
   result on the host), so it must not be called while its stream -- or, in global capture
   mode, any stream -- is being captured. Returns iterations or -1 as conj_grad does, -2 for
   unsupported arguments (including pointers that are not memory of the current device),
   -3 if the solver aborted, -4 if the work area's address is unavailable, -5 for a CUDA
   error already pending or in reading the result; a kernel that cannot be launched ends
   the process, as elsewhere in this library. precond: 0 implicit Jacobi, 1 Jacobi. */
int mzb_conj_grad_noalloc(const double *b, const double *x0, double *x, double tol, int n,
                          int precond, void *stream);

/* Several resident systems. No counterpart in the reference, which holds one global
   system per process (library/src/solver_md.c:12-14); every reference call above acts on
   the selected system. mzb_system_create makes a new empty system and selects it
   (initialise it with solver_initialize, solver_initialize_grid, ...); select/destroy
   return -1 for an unknown handle. */
int mzb_system_create(void);
int mzb_system_select(int handle);
int mzb_system_current(void);
int mzb_system_destroy(int handle);

/* Advance the listed systems by n_steps MD steps (solver.py:483-492 each) together: one
   CUDA graph per step, whose branches run each system's integrator, charge spreading and
   forces, and one cooperative launch that runs every system's field solve on its own
   range of CTAs. Every system must be initialised, bootstrapped and use the FP32+refine
   field solve (mzb_set_precision(1, ...)). Charge errors exit as solver_update_charges
   does, after the call. Returns 0, or -1 if a field solve did not converge. No
   counterpart in the reference. */
int mzb_batch_step(const int *handles, int nsys, int n_steps);

/* Size classes side by side: system r belongs to class cls[r]; class c advances
   class_steps[c] MD steps on its own stream while the others run, its systems' field
   solves sharing class_ctas[c] CTAs (at least one per system; the counts add up to at
   most the SM count). Each class takes the steps of mzb_batch_step, with the same
   results. Returns when all classes are done: 0, or -1 if a field solve did not
   converge. No counterpart in the reference. */
int mzb_batch_classes(const int *handles, const int *cls, int nsys, const int *class_ctas,
                      const int *class_steps, int nclass);

/* Tune the batched field solve on the listed systems, timing batched solves of every
   system's current charges from its previous field (an MD-step update): per size class
   (systems of one grid size) alone, each distinct coarse-level plan (mzb_set_mixed_plan),
   keeping the fastest and its time per grid point; then, on the whole set, team partitions
   with CTAs per system ~ grid points^alpha x that class time per point (alpha in {1.2, 1.0,
   0.8, 0.6, 0.4}), keeping the fastest; and the pair forces. out[0..3] = {partition
   exponent, pair-force CTAs, solve ms, forces ms}. Leaves the systems' state unchanged
   except for the plans and shares chosen. */
int mzb_batch_autotune(const int *handles, int nsys, double *out);

/* Device bytes one FP32+refine system with an n^3 grid and n_p ions holds (admission
   against an HBM budget). */
double mzb_system_footprint(int n, int n_p);

/* Release the device blocks the library keeps for reuse after systems are finalised (a
   later system of the same sizes takes them instead of new allocations); returns the
   bytes released. */
size_t mzb_trim_device_cache(void);

/* Asynchronous output snapshots of the selected system (the reference's output path,
   maze_poisson/myio/output/csv.py:45-183, calls the blocking getters every stride).
   begin stages the requested arrays on the system's stream and copies them to pinned
   host memory on a copy stream, overlapping the next MD steps; it returns the slot (0 or
   1), or -1 when both slots hold unfetched snapshots. what: 1 positions, 2 velocities,
   4 forces (elec, noel, tot), 8 scalars {q total, V_notelec, K, Px, Py, Pz, T, 0},
   16 fields (phi, phi_prev). fetch waits for the slot, copies into the given arrays
   (null skips one) and frees the slot; it returns the captured mask or -1. */
int mzb_snapshot_begin(int what);
int mzb_snapshot_fetch(int slot, double *pos, double *vel, double *fcs_elec, double *fcs_noel,
                       double *fcs_tot, double *scalars, double *phi, double *phi_prev);
/* The slot's pinned host buffer, read in place without a copy (layout: pos, vel,
   fcs_elec, fcs_noel, fcs_tot as n_p*3 doubles each, 8 scalars, then phi, phi_prev as
   n^3 each when captured), after waiting for it; valid until mzb_snapshot_fetch releases
   the slot. Null if the slot holds no snapshot. */
double *mzb_snapshot_host(int slot);

/* instrumentation */
void *mzb_get_stream(void);                /* cudaStream_t of the current system */
double mzb_last_solve_ms(void);            /* device ms of the last field-solver launch */
int mzb_last_solve_result(void);           /* its return value (iterations or -1) */
uint64_t mzb_kernel_launches(void);        /* kernels this library has launched */
int mzb_sm_count(void);                    /* SMs of the current device (CTA shares of the batched step) */
/* Green's function of the unscaled periodic 7-point Laplacian on an n^3 grid (2 <= n <= 16),
   g[d] = (1/n^3) sum_{k != 0} cos(2 pi k.d / n) / lambda(k): the mixed solver's exact
   coarsest-level solve. Host-only; returns 0, or -1 for an n out of range. */
int mzb_coarse_green(int n, float *g);

#ifdef __cplusplus
}
#endif

#endif /* MAZE_POISSON_B200_H */
