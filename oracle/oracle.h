/*
 * CPU oracle for the MaZe_Poisson per-step MD hot path -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of the reference library's FP64 algorithm (MaZe_Poisson,
 * library/src), used by tests/, __graft_entry__.smoke() and bench.py's cpu_baseline
 * leg as the checker. It is never linked into, imported by, or called from the product
 * (maze_poisson_b200/). It exports the same facade symbols as the reference's
 * libmaze_poisson.so (library/src/solver_md.c) so that one ctypes binding drives the
 * product, this oracle and the compiled reference alike, plus a few kernel-level
 * functions (prefixed `orc_`) with the reference's argument meaning but plain
 * (halo-free) n^3 arrays.
 *
 * Every operation keeps the reference's evaluation order and uses no fused
 * multiply-add, so that with OMP_NUM_THREADS=1 the results are bit-identical to the
 * reference's parity build (oracle/Makefile `ref`); tests/test_oracle_pin.py checks this
 * against golden vectors made by the compiled reference (tests/golden/make_golden.py).
 * The FFT Poisson path is restated in numpy (oracle/fft_oracle.py): its arithmetic lives
 * in FFTW3, which the reference does not vendor.
 */
#ifndef MAZE_ORACLE_H
#define MAZE_ORACLE_H

#include <stdint.h>

/* grid kernels on n^3 periodic arrays, idx = (i*n + j)*n + k */
void orc_laplace(const double *u, double *out, int n);                       /* laplace.c:24-75 */
int orc_conj_grad(const double *b, const double *x0, double *x, double tol, int n); /* plcg.c:28-90 */
void orc_smooth_rbgs(const double *rhs, double *x, int n, int iters);          /* multigrid.c:636-729 */
void orc_restrict27(const double *fine, double *coarse, int n);                /* multigrid.c:523-594 */
void orc_prolong_trilinear(const double *coarse, double *fine, int nc);        /* multigrid.c:393-463 */
int orc_cg_coarse(const double *b, double *x, int n, int maxit, double rtol);  /* multigrid.c:13-96 */
void orc_mg_apply(const double *rhs, double *x, int n, int sm);                /* multigrid.c:99-168,743 */

void orc_ssor_apply(const double *in, double *out, int n);                      /* precond_ssor.c:1240-1252 */
void orc_blockjacobi_apply(const double *in, double *out, int n);          /* precond_blockjacobi.c:173-206 */
void orc_blockjacobi_inverse(double *out);                                  /* precond_blockjacobi.c:14-69 */

/* Poisson-Boltzmann kernels on n^3 arrays: ex/ey/ez are the +x/+y/+z face dielectric
   coefficients of each point, k2 its screening term */
void orc_update_eps_k2(const double *pos, const double *radii, int np, int n, double h, double w,
                       double eps_s, double eps_int, double kbar2, double *eps_x, double *eps_y,
                       double *eps_z, double *k2);                                     /* grid_general.c:138-301 */
void orc_laplace_pb(const double *u, double *out, const double *ex, const double *ey,
                    const double *ez, const double *k2, int n);                        /* laplace.c:77-145 */
int orc_conj_grad_pb(const double *b, const double *x0, double *x, double tol, int n,
                     const double *ex, const double *ey, const double *ez, const double *k2); /* plcg.c:169-238 */
void orc_smooth_pb(const double *rhs, double *x, int n, int iters, const double *ex,
                   const double *ey, const double *ez, const double *k2);          /* multigrid_pb.c:544-640 */
void orc_restrict_eps(const double *in, double *out, int n, int axis);              /* multigrid_pb.c:330-447 */
void orc_restrict_k2(const double *in, double *out, int n);                         /* multigrid_pb.c:459-527 */
int orc_cg_coarse_pb(const double *b, double *x, int n, int maxit, double rtol, const double *ex,
                     const double *ey, const double *ez, const double *k2);        /* multigrid_pb.c:16-97 */
void orc_mg_pb_apply(const double *rhs, double *x, int n, int sm, const double *ex,
                     const double *ey, const double *ez, const double *k2);        /* multigrid_pb.c:270-328 */
void orc_forces_pb(const double *pos, const double *radii, int np, int n, double h, double w,
                   double eps_s, double eps_int, double gamma_np, int nonpolar, const double *phi,
                   const double *ex, const double *ey, const double *ez, const double *k2,
                   double *fdb, double *fib, double *fnp);                          /* particles.c:420-775 */
void orc_get_pb_grids(double *ex, double *ey, double *ez, double *k2);

/* particle kernels */
void orc_cic_neighbors(const double *pos, int np, int n, double h, int64_t *nbr);      /* particles.c:297-346 */
void orc_spline_neighbors(const double *pos, int np, int n, double h, int64_t *nbr);   /* particles.c:348-385 */
/* spreading / field force for scheme cas (0 CIC, 1 SPL_QUADR, 2 SPL_CUBIC; charges.c:8-38,
   100-144, forces.c:26-100); nbr_out (np * points * 3) receives the neighbour list if set */
double orc_spread_scheme(const double *pos, const double *chg, int np, int n, double h, int cas,
                         double *q, int64_t *nbr_out);
double orc_force_scheme(const double *phi, const double *chg, const double *pos, int np, int n,
                        double h, int cas, double *f);
double orc_spread_cic(const double *pos, const double *chg, const int64_t *nbr, int np,
                      int n, double h, double *q);                                       /* charges.c:100-144 */
double orc_force_fd(const double *phi, const int64_t *nbr, const double *chg,
                    const double *pos, int np, int n, double h, double *f);               /* forces.c:26-100 */
double orc_tf_forces(const double *pos, const int32_t *types, const double *tab, int ntyp,
                     int np, double L, double rcut, double *f);                           /* forces.c:112-186 */
void orc_tf_table(const double *pot_params, int ntyp, double L, double *tab);             /* particles.c:181-228 */
void orc_lj_table(const double *pot_params, int ntyp, double L, double *tab);             /* particles.c:230-266 */
double orc_lj_forces(const double *pos, const int32_t *types, const double *tab, int ntyp, int np,
                     double L, double rcut, double *f);                                    /* forces.c:199-271 */
void orc_sc_table(const double *pot_params, int ntyp, double L, double *tab);             /* particles.c:268-295 */
double orc_sc_forces(const double *pos, const double *tab, int np, double L, double rcut,
                     double *f);                                                           /* forces.c:283-337 */
void orc_cell_list(const double *pos, int np, double L, int nc, int32_t *cell_start,
                   int32_t *cell_ions);                                                   /* linkedcell.py:4-53 */

/* facade with the reference's exported names (solver_md.c:19-354) */
void solver_initialize(void);
void solver_initialize_grid(int n, double L, double h, double tol, double eps_s, double eps_int,
                            int grid_type, int precond_type);
void solver_initialize_particles(int n, int n_typ, double L, double h, int n_p, int pot_type,
                                 int cas_type, int *types, double *pos, double *vel, double *mass,
                                 double *charges, double *pot_params);
void solver_initialize_integrator(int n_p, double dt, double T, double gamma, int itg_type,
                                  int itg_enabled);
int solver_update_charges(void);
void solver_init_field(void);
int solver_update_field(void);
void solver_set_field(double *phi);
void solver_set_field_prev(double *phi);
void solver_compute_forces_elec(void);
double solver_compute_forces_noel(void);
void solver_compute_forces_tot(void);
void integrator_part_1(void);
void integrator_part_2(void);
int solver_check_thermostat(void);
void solver_rescale_velocities(void);
void solver_finalize(void);
void solver_initialize_grid_pois_boltz(double w, double kbar2, int nonpolar);
void solver_initialize_particles_pois_boltz(double gamma_np, double beta_np, double *radii);
void solver_update_eps_k2(void);
double solver_compute_forces_pb(void);
void get_fcs_db(double *o);
void get_fcs_ib(double *o);
void get_fcs_np(double *o);
void get_radii(double *o);

void get_pos(double *o);
void get_vel(double *o);
void get_fcs_elec(double *o);
void get_fcs_noel(double *o);
void get_fcs_tot(double *o);
void get_field(double *o);
void get_field_prev(double *o);
void get_q(double *o);
double get_kinetic_energy(void);
double get_temperature(void);
void get_momentum(double *o);

/* OVRVO noise injection: the next O-block draws its N(0,1) variates from this buffer
   (3*n_p values per O-block, consumed in order) instead of an RNG. */
void orc_set_noise(const double *z, int64_t count);

#endif
