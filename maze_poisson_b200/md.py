"""MD driver over the C ABI, mirroring the reference's SolverMD call sequence.

`MDRun` makes the same ctypes calls, in the same order, as maze_poisson/solver.py:
initialize (96-108), the two bootstrap Verlet steps of initialize_md (371-409) and
md_loop_iter (483-492) -- so it drives this build's libmaze_poisson.so exactly the way
the reference's solver.py would, without the reference's file I/O.
"""
import numpy as np

from .systems import T_AU_FS


def gamma_au(gamma_per_ps):
    """Langevin friction in a.u.^-1 from ps^-1 (the reference takes `gamma` in a.u.)."""
    return gamma_per_ps * 1e-3 * T_AU_FS


class MDRun:
    def __init__(self, capi, system, method="LCG", precond="NONE", tol=1e-7, integrator="VERLET",
                 thermostat=False, T=1200.0, gamma_per_ps=1.0, dt_fs=1.0, eps_s=1.0, eps_int=1.0,
                 rescale=False, precision=0, mixed_tol=0.0, cas="CIC", pot="TF", pb=None):
        self.capi = capi
        self.sys = system
        self.method = method.upper()
        self.precond = precond.upper()
        self.tol = tol
        self.integrator = integrator.upper()
        self.thermostat = thermostat
        self.T = T
        self.gamma = gamma_au(gamma_per_ps)
        self.dt = dt_fs / T_AU_FS
        self.eps_s = eps_s
        self.eps_int = eps_int
        self.rescale = rescale
        self.cas = cas.upper()  # charge assignment: CIC, SPL_QUADR, SPL_CUBIC
        self.pot = pot.upper()  # pair potential: TF, LJ, SC (system.pot_params to match)
        # field-solve precision (this build's extension): 0 FP64 reference algorithms,
        # 1 FP32 multigrid + FP64 refinement to mixed_tol (or tol when 0), 2 the same
        # multigrid and refinement with every value in FP64
        self.precision = precision
        self.mixed_tol = mixed_tol
        # Poisson-Boltzmann implicit solvent (systems.PBSettings) or None
        self.pb = pb
        self.n_iters = None
        self.potential_notelec = None

    # -- solver.py:96-108 + initialize_md 371-409 -------------------------------------
    def initialize(self):
        c = self.capi
        s = self.sys
        c.solver_initialize()
        maps = c.type_maps()
        c.solver_initialize_grid(s.n_grid, s.L, s.h, self.tol, self.eps_s, self.eps_int,
                                 maps["method"][self.method], maps["precond"][self.precond])
        if self.pb is not None:  # solver.py:145-163
            c.solver_initialize_grid_pois_boltz(self.pb.w, self.pb.kbar2, int(self.pb.nonpolar))
        if self.precision:
            c.mzb_set_precision(int(self.precision), float(self.mixed_tol))
        c.solver_initialize_particles(s.n_grid, 2, s.L, s.h, s.n_ions, maps["potential"][self.pot],
                                      maps["cas"][self.cas], s.types, s.pos, s.vel, s.mass, s.charges,
                                      s.pot_params)
        if self.pb is not None:  # solver.py:346-356
            c.solver_initialize_particles_pois_boltz(self.pb.gamma_np, self.pb.beta_np, self.pb.radii)
        c.solver_initialize_integrator(s.n_ions, self.dt, self.T, self.gamma,
                                       maps["integrator"][self.integrator], 1 if self.thermostat else 0)
        # step 0
        self.update_charges()
        c.solver_init_field()
        self.compute_forces()
        # step 1
        c.integrator_part_1()
        self.update_charges()
        c.solver_init_field()
        self.compute_forces()
        c.integrator_part_2()
        if self.rescale:
            c.solver_rescale_velocities()

    # -- solver.py:371-409 with a restart field -------------------------------------------
    def restart(self, pos, vel, field, field_prev):
        """Start from a saved state the way the reference's restart path does: the particles
        from the restart positions and velocities, solver_set_field / solver_set_field_prev
        in place of the two bootstrap steps; then the forces of that state are computed,
        so that the first step integrates with them."""
        c = self.capi
        s = self.sys
        s.pos = np.ascontiguousarray(pos, dtype=np.float64)
        s.vel = np.ascontiguousarray(vel, dtype=np.float64)
        c.solver_initialize()
        maps = c.type_maps()
        c.solver_initialize_grid(s.n_grid, s.L, s.h, self.tol, self.eps_s, self.eps_int,
                                 maps["method"][self.method], maps["precond"][self.precond])
        if self.pb is not None:
            c.solver_initialize_grid_pois_boltz(self.pb.w, self.pb.kbar2, int(self.pb.nonpolar))
        if self.precision:
            c.mzb_set_precision(int(self.precision), float(self.mixed_tol))
        c.solver_initialize_particles(s.n_grid, 2, s.L, s.h, s.n_ions, maps["potential"][self.pot],
                                      maps["cas"][self.cas], s.types, s.pos, s.vel, s.mass, s.charges,
                                      s.pot_params)
        if self.pb is not None:
            c.solver_initialize_particles_pois_boltz(self.pb.gamma_np, self.pb.beta_np, self.pb.radii)
        c.solver_initialize_integrator(s.n_ions, self.dt, self.T, self.gamma,
                                       maps["integrator"][self.integrator], 1 if self.thermostat else 0)
        self.update_charges()
        c.solver_set_field(np.ascontiguousarray(field, dtype=np.float64))
        c.solver_set_field_prev(np.ascontiguousarray(field_prev, dtype=np.float64))
        self.compute_forces()

    def update_charges(self):
        if self.capi.solver_update_charges() != 0:
            raise RuntimeError("charge is not preserved")
        if self.pb is not None:  # solver.py:411-415, called after every charge update
            self.capi.solver_update_eps_k2()

    def compute_forces(self):
        c = self.capi
        c.solver_compute_forces_elec()
        self.potential_notelec = c.solver_compute_forces_noel()
        if self.pb is not None:
            self.energy_nonpolar = c.solver_compute_forces_pb()
        c.solver_compute_forces_tot()

    # -- solver.py:483-492 --------------------------------------------------------------
    def step(self):
        c = self.capi
        c.integrator_part_1()
        self.update_charges()
        self.n_iters = c.solver_update_field()
        self.compute_forces()
        c.integrator_part_2()
        return self.n_iters

    def run(self, n_steps):
        for _ in range(n_steps):
            self.step()

    # -- getters (solver_md.c:247-354) ---------------------------------------------------
    def state(self, fields=True):
        c = self.capi
        n = self.sys.n_ions
        out = {}
        names = ("pos", "vel", "fcs_elec", "fcs_noel", "fcs_tot")
        if self.pb is not None:
            names += ("fcs_db", "fcs_ib", "fcs_np")
        for name in names:
            a = np.empty((n, 3), dtype=np.float64)
            getattr(c, "get_" + name)(a)
            out[name] = a
        if fields:
            g = self.sys.n_grid
            for name in ("field", "field_prev", "q"):
                a = np.empty((g, g, g), dtype=np.float64)
                getattr(c, "get_" + name)(a)
                out[name] = a
        out["kinetic"] = c.get_kinetic_energy()
        out["potential_notelec"] = self.potential_notelec
        out["n_iters"] = self.n_iters
        return out

    def finalize(self):
        self.capi.solver_finalize()
