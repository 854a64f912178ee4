"""The drop-in boundary: the built library loads and exports every symbol declared in
include/*.h, the binding covers the reference's registrations, and the enum tables match
the reference's strings. No GPU work is launched here."""
import ctypes
import glob
import os
import re

from conftest import ROOT
from maze_poisson_b200.c_api import EXTENSION_SYMBOLS, REFERENCE_SYMBOLS, CAPI

DECL = re.compile(r"^\s*(?:int|void|double|char\s*\*|uint64_t|size_t)\s*\*?\s*([a-z_0-9]+)\s*\(", re.M)


def declared():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        names |= set(DECL.findall(open(h).read()))
    return names


def test_headers_declare_binding():
    d = declared()
    assert set(REFERENCE_SYMBOLS) <= d
    assert set(EXTENSION_SYMBOLS) <= d


def test_library_exports_every_declared_symbol(product_path):
    lib = ctypes.CDLL(product_path, mode=ctypes.RTLD_LOCAL)
    missing = [n for n in sorted(declared()) if not hasattr(lib, n)]
    assert not missing, missing


def test_enum_tables_match_reference(product_path):
    c = CAPI(product_path)
    m = c.type_maps()
    assert m["method"] == {"LCG": 0, "FFT": 1, "MULTIGRID": 2, "MAZE-LCG": 3, "MAZE-MULTIGRID": 4}
    assert m["precond"] == {"NONE": 0, "JACOBI": 1, "MG": 2, "SSOR": 3, "BLOCKJACOBI": 4}
    assert m["potential"] == {"TF": 0, "LJ": 1, "SC": 2}
    assert m["cas"] == {"CIC": 0, "SPL_QUADR": 1, "SPL_CUBIC": 2}
    assert m["integrator"] == {"OVRVO": 0, "VERLET": 1}
    assert c.init_mpi() == 0 and c.get_rank() == 0


def test_reference_binding_signatures_cover_ctypes_layer():
    """Every name the reference's c_api registers is bound here with a restype."""
    ref_names = {
        "solver_initialize", "solver_initialize_grid", "solver_initialize_grid_pois_boltz",
        "solver_initialize_particles", "solver_initialize_particles_pois_boltz",
        "solver_initialize_integrator", "solver_update_charges", "solver_init_field",
        "solver_set_field", "solver_set_field_prev", "solver_update_field", "solver_update_eps_k2",
        "solver_compute_forces_elec", "solver_compute_forces_noel", "solver_compute_forces_pb",
        "solver_compute_forces_tot", "integrator_part_1", "integrator_part_2",
        "solver_check_thermostat", "solver_rescale_velocities", "solver_finalize",
        "get_grid_type_num", "get_grid_type_str", "get_potential_type_num", "get_potential_type_str",
        "get_ca_scheme_type_num", "get_ca_scheme_type_str", "get_integrator_type_num",
        "get_integrator_type_str", "get_precond_type_num", "get_precond_type_str", "get_pos",
        "get_vel", "get_fcs_elec", "get_fcs_noel", "get_fcs_db", "get_fcs_ib", "get_fcs_np",
        "get_fcs_tot", "get_charges", "get_types", "get_masses", "get_radii", "get_field",
        "get_field_prev", "get_q", "get_kinetic_energy", "get_energy_elec", "get_momentum",
        "get_temperature", "init_mpi", "get_rank"}
    assert ref_names == set(REFERENCE_SYMBOLS)
