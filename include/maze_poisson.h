/*
 * libmaze_poisson.so -- B200 (sm_100a) drop-in for MaZe_Poisson's native library.
 *
 * Every function below replaces the reference function of the same name; the
 * reference's Python layer binds them through ctypes with the argtypes of
 * maze_poisson/c_api/{solver,get_functions,mpi_base}.py. One global MD system lives
 * on the GPU (the reference's g_grid/g_particles/g_integrator singletons,
 * library/src/solver_md.c:12-14); all arrays crossing this boundary are caller-owned
 * host buffers, copied in by the initialisers/setters and out by the getters.
 * Not reentrant; call from one thread. Fatal conditions print and exit(1) where the
 * reference does. Extensions of this build are in maze_poisson_b200.h.
 */
#ifndef MAZE_POISSON_H
#define MAZE_POISSON_H

#ifdef __cplusplus
extern "C" {
#endif

/* serial MPI stubs: library/src/mpi_base.c:169-177 (init_mpi), :18-20 (get_rank);
   bound at maze_poisson/c_api/mpi_base.py:8-9 */
int init_mpi(void);
int get_rank(void);

/* enum <-> name tables: grid_general.c:8-22, particles.c:17-36, integrator_general.c:7-15 */
int get_grid_type_num(void);
char *get_grid_type_str(int n);
int get_precond_type_num(void);
char *get_precond_type_str(int n);
int get_potential_type_num(void);
char *get_potential_type_str(int n);
int get_ca_scheme_type_num(void);
char *get_ca_scheme_type_str(int n);
int get_integrator_type_num(void);
char *get_integrator_type_str(int n);

/* lifecycle and set-up: solver_md.c:19-89 */
void solver_initialize(void);
void solver_initialize_grid(int n_grid, double L, double h, double tol, double eps,
                            double eps_int, int grid_type, int precond_type);
void solver_initialize_grid_pois_boltz(double w, double kbar2, int nonpolar_enabled);
void solver_initialize_particles(int n, int n_typ, double L, double h, int n_p, int pot_type,
                                 int cas_type, int *types, double *pos, double *vel, double *mass,
                                 double *charges, double *pot_params);
void solver_initialize_particles_pois_boltz(double gamma_np, double beta_np, double *solv_radii);
void solver_initialize_integrator(int n_p, double dt, double T, double gamma, int itg_type,
                                  int itg_enabled);

/* the per-step hot path: solver_md.c:91-184 */
int solver_update_charges(void);          /* solver_md.c:91-107: CIC spread + charge check */
void solver_init_field(void);              /* solver_md.c:109-111 */
void solver_set_field(double *phi);        /* solver_md.c:113-119 */
void solver_set_field_prev(double *phi);   /* solver_md.c:121-129 */
int solver_update_field(void);             /* solver_md.c:131-133: iterations or -1 */
void solver_update_eps_k2(void);           /* solver_md.c:135-138 (Poisson-Boltzmann) */
void solver_compute_forces_elec(void);     /* solver_md.c:140-142 */
double solver_compute_forces_noel(void);   /* solver_md.c:144-146: returns V_notelec */
double solver_compute_forces_pb(void);     /* solver_md.c:148-150 (Poisson-Boltzmann) */
void solver_compute_forces_tot(void);      /* solver_md.c:152-154 */
void integrator_part_1(void);              /* solver_md.c:162-164 */
void integrator_part_2(void);              /* solver_md.c:166-168 */
int solver_check_thermostat(void);         /* solver_md.c:210-221 */
void solver_rescale_velocities(void);      /* solver_md.c:170-172 */
void solver_finalize(void);                /* solver_md.c:230-245 */

/* getters: solver_md.c:247-354 (caller-owned C-contiguous buffers) */
void get_pos(double *recv);
void get_vel(double *recv);
void get_fcs_elec(double *recv);
void get_fcs_noel(double *recv);
void get_fcs_db(double *recv);
void get_fcs_ib(double *recv);
void get_fcs_np(double *recv);
void get_fcs_tot(double *recv);
void get_types(int *recv);
void get_charges(double *recv);
void get_masses(double *recv);
void get_radii(double *recv);
void get_field(double *recv);
void get_field_prev(double *recv);
void get_q(double *recv);
double get_kinetic_energy(void);
double get_energy_elec(void);
void get_momentum(double *recv);
double get_temperature(void);

#ifdef __cplusplus
}
#endif

#endif /* MAZE_POISSON_H */
