"""ctypes binding of libmaze_poisson.so, mirroring the reference's maze_poisson/c_api.

Every symbol is registered with the argtypes/restype that the reference registers
(maze_poisson/c_api/solver.py:8-176, get_functions.py:9-194, mpi_base.py:8-9), so the
same calls -- and the same numpy buffers -- drive this library, or any library with the
reference's ABI. Extensions of this build (no reference counterpart) are registered
too and declared in include/maze_poisson_b200.h.

Unlike the reference's `SafeCallable`, which logs and calls exit() on a missing symbol,
this binding raises at load time: a product library without its symbols must fail
loudly.
"""
import ctypes
import os

import numpy as np
import numpy.ctypeslib as npct

from . import library_path

_i32_1 = npct.ndpointer(dtype=np.int32, ndim=1, flags="C_CONTIGUOUS")
_f64_1 = npct.ndpointer(dtype=np.float64, ndim=1, flags="C_CONTIGUOUS")
_f64_2 = npct.ndpointer(dtype=np.float64, ndim=2, flags="C_CONTIGUOUS")
_f64_3 = npct.ndpointer(dtype=np.float64, ndim=3, flags="C_CONTIGUOUS")
_i64_3 = npct.ndpointer(dtype=np.int64, ndim=3, flags="C_CONTIGUOUS")
_f64_any = npct.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")

_c = ctypes
# name -> (restype, argtypes): the reference's registrations
REFERENCE_SYMBOLS = {
    "init_mpi": (_c.c_int, []),
    "get_rank": (_c.c_int, []),
    "solver_initialize": (None, []),
    "solver_initialize_grid": (None, [_c.c_int, _c.c_double, _c.c_double, _c.c_double, _c.c_double,
                                      _c.c_double, _c.c_int, _c.c_int]),
    "solver_initialize_grid_pois_boltz": (None, [_c.c_double, _c.c_double, _c.c_int]),
    "solver_initialize_particles": (None, [_c.c_int, _c.c_int, _c.c_double, _c.c_double, _c.c_int,
                                           _c.c_int, _c.c_int, _i32_1, _f64_2, _f64_2, _f64_1, _f64_1,
                                           _f64_1]),
    "solver_initialize_particles_pois_boltz": (None, [_c.c_double, _c.c_double, _f64_1]),
    "solver_initialize_integrator": (None, [_c.c_int, _c.c_double, _c.c_double, _c.c_double, _c.c_int,
                                            _c.c_int]),
    "solver_update_charges": (_c.c_int, []),
    "solver_init_field": (None, []),
    "solver_set_field": (None, [_f64_3]),
    "solver_set_field_prev": (None, [_f64_3]),
    "solver_update_field": (_c.c_int, []),
    "solver_update_eps_k2": (None, []),
    "solver_compute_forces_elec": (None, []),
    "solver_compute_forces_noel": (_c.c_double, []),
    "solver_compute_forces_pb": (_c.c_double, []),
    "solver_compute_forces_tot": (None, []),
    "integrator_part_1": (None, []),
    "integrator_part_2": (None, []),
    "solver_check_thermostat": (_c.c_int, []),
    "solver_rescale_velocities": (None, []),
    "solver_finalize": (None, []),
    "get_grid_type_num": (_c.c_int, []),
    "get_grid_type_str": (_c.c_char_p, [_c.c_int]),
    "get_potential_type_num": (_c.c_int, []),
    "get_potential_type_str": (_c.c_char_p, [_c.c_int]),
    "get_ca_scheme_type_num": (_c.c_int, []),
    "get_ca_scheme_type_str": (_c.c_char_p, [_c.c_int]),
    "get_integrator_type_num": (_c.c_int, []),
    "get_integrator_type_str": (_c.c_char_p, [_c.c_int]),
    "get_precond_type_num": (_c.c_int, []),
    "get_precond_type_str": (_c.c_char_p, [_c.c_int]),
    "get_pos": (None, [_f64_2]),
    "get_vel": (None, [_f64_2]),
    "get_fcs_elec": (None, [_f64_2]),
    "get_fcs_noel": (None, [_f64_2]),
    "get_fcs_db": (None, [_f64_2]),
    "get_fcs_ib": (None, [_f64_2]),
    "get_fcs_np": (None, [_f64_2]),
    "get_fcs_tot": (None, [_f64_2]),
    "get_charges": (None, [_f64_1]),
    "get_types": (None, [_i32_1]),
    "get_masses": (None, [_f64_1]),
    "get_radii": (None, [_f64_1]),
    "get_field": (None, [_f64_3]),
    "get_field_prev": (None, [_f64_3]),
    "get_q": (None, [_f64_3]),
    "get_kinetic_energy": (_c.c_double, []),
    "get_energy_elec": (_c.c_double, []),
    "get_momentum": (None, [_f64_1]),
    "get_temperature": (_c.c_double, []),
}

# Extensions of this build (include/maze_poisson_b200.h).
EXTENSION_SYMBOLS = {
    "solver_md_step": (_c.c_int, [_c.c_int]),
    "mzb_laplace": (None, [_f64_any, _f64_any, _c.c_int]),
    "mzb_conj_grad": (_c.c_int, [_f64_any, _f64_any, _f64_any, _c.c_double, _c.c_int, _c.c_int]),
    "mzb_smooth_rbgs": (None, [_f64_any, _f64_any, _c.c_int, _c.c_int]),
    "mzb_restrict27": (None, [_f64_any, _f64_any, _c.c_int]),
    "mzb_prolong_trilinear": (None, [_f64_any, _f64_any, _c.c_int]),
    "mzb_cg_coarse": (_c.c_int, [_f64_any, _f64_any, _c.c_int, _c.c_int, _c.c_double]),
    "mzb_mg_apply": (None, [_f64_any, _f64_any, _c.c_int, _c.c_int]),
    "mzb_ssor_apply": (None, [_f64_any, _f64_any, _c.c_int]),
    "mzb_blockjacobi_apply": (None, [_f64_any, _f64_any, _c.c_int]),
    "mzb_laplace_pb": (None, [_f64_any] * 6 + [_c.c_int]),
    "mzb_conj_grad_pb": (_c.c_int, [_f64_any, _f64_any, _f64_any, _c.c_double, _c.c_int] + [_f64_any] * 4),
    "mzb_smooth_pb": (None, [_f64_any, _f64_any, _c.c_int, _c.c_int] + [_f64_any] * 4),
    "mzb_mg_pb_apply": (None, [_f64_any, _f64_any, _c.c_int, _c.c_int] + [_f64_any] * 4),
    "mzb_restrict_pb": (None, [_f64_any] * 8 + [_c.c_int]),
    "mzb_get_pb_grids": (None, [_f64_any] * 4),
    "mzb_fft_poisson": (None, [_f64_any, _f64_any, _c.c_int, _c.c_double, _c.c_double]),
    "mzb_get_cic_neighbors": (None, [_i64_3]),
    "mzb_set_cell_grid": (None, [_c.c_int]),
    "mzb_get_cells": (_c.c_int, [_i32_1, _i32_1]),
    "mzb_philox_normals": (None, [_c.c_uint64, _f64_2]),
    "mzb_set_seed": (None, [_c.c_uint64]),
    "mzb_get_ocalls": (_c.c_uint64, []),
    "mzb_get_stream": (_c.c_void_p, []),
    "mzb_last_solve_ms": (_c.c_double, []),
    "mzb_last_solve_result": (_c.c_int, []),
    "mzb_kernel_launches": (_c.c_uint64, []),
    "mzb_sm_count": (_c.c_int, []),
    "mzb_coarse_green": (_c.c_int, [_c.c_int, _c.c_void_p]),
    "mzb_set_precision": (None, [_c.c_int, _c.c_double]),
    "mzb_get_precision": (_c.c_int, []),
    "mzb_set_mixed_plan": (_c.c_int, [_c.c_int]),
    "mzb_get_mixed_plan": (_c.c_int, []),
    "mzb_set_mixed_sweeps": (_c.c_int, [_c.c_int, _c.c_int]),
    "mzb_get_mixed_sweeps": (None, [_c.POINTER(_c.c_int), _c.POINTER(_c.c_int)]),
    "mzb_conj_grad_noalloc": (_c.c_int, [_c.c_void_p, _c.c_void_p, _c.c_void_p, _c.c_double, _c.c_int,
                                         _c.c_int, _c.c_void_p]),
    "mzb_system_create": (_c.c_int, []),
    "mzb_system_select": (_c.c_int, [_c.c_int]),
    "mzb_system_current": (_c.c_int, []),
    "mzb_system_destroy": (_c.c_int, [_c.c_int]),
    "mzb_batch_step": (_c.c_int, [_i32_1, _c.c_int, _c.c_int]),
    "mzb_batch_classes": (_c.c_int, [_i32_1, _i32_1, _c.c_int, _i32_1, _i32_1, _c.c_int]),
    "mzb_batch_autotune": (_c.c_int, [_i32_1, _c.c_int, _f64_1]),
    "mzb_system_footprint": (_c.c_double, [_c.c_int, _c.c_int]),
    "mzb_trim_device_cache": (_c.c_size_t, []),
    "mzb_snapshot_begin": (_c.c_int, [_c.c_int]),
    "mzb_snapshot_fetch": (_c.c_int, [_c.c_int] + [_c.c_void_p] * 8),
    "mzb_snapshot_host": (_c.POINTER(_c.c_double), [_c.c_int]),
}


class CAPI:
    """Bound functions of one shared library with the reference's C ABI.

    `CAPI()` loads this build's libmaze_poisson.so; `CAPI(path, extensions=False)` loads
    any other library with the reference's ABI (only the reference symbols are bound).
    The reference holds one global MD system; this build holds several (mzb_system_*),
    and the reference calls act on the selected one.
    """

    def __init__(self, path=None, extensions=True, mode=ctypes.RTLD_LOCAL):
        self.path = os.path.abspath(path or library_path(require=True))
        self.library = ctypes.CDLL(self.path, mode=mode)
        table = dict(REFERENCE_SYMBOLS)
        if extensions:
            table.update(EXTENSION_SYMBOLS)
        self.functions = {}
        for name, (restype, argtypes) in table.items():
            try:
                fn = getattr(self.library, name)
            except AttributeError as e:
                raise RuntimeError(f"{self.path} does not export {name}") from e
            fn.restype = restype
            fn.argtypes = argtypes
            self.functions[name] = fn

    def __getattr__(self, name):
        fns = self.__dict__.get("functions", {})
        if name in fns:
            return fns[name]
        raise AttributeError(name)

    def type_maps(self):
        """Name -> enum maps read from the library (maze_poisson/solver.py:115-127)."""
        maps = {}
        for key, fnum, fstr in [("method", "get_grid_type_num", "get_grid_type_str"),
                                ("potential", "get_potential_type_num", "get_potential_type_str"),
                                ("cas", "get_ca_scheme_type_num", "get_ca_scheme_type_str"),
                                ("integrator", "get_integrator_type_num", "get_integrator_type_str"),
                                ("precond", "get_precond_type_num", "get_precond_type_str")]:
            n = getattr(self, fnum)()
            maps[key] = {getattr(self, fstr)(i).decode("utf-8").upper(): i for i in range(n)}
        return maps
