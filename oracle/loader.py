"""Build and load the oracle libraries -- TEST INFRASTRUCTURE ONLY.

liboracle.so is the CPU restatement (oracle.c); _ref/libmaze_poisson_ref*.so are the
reference's own C sources compiled by oracle/Makefile (only where the reference tree is
present; the built files travel with the working tree). Only tests/, the smoke check and
bench.py's CPU-baseline leg use this module.
"""
import ctypes
import os
import subprocess

import numpy as np
import numpy.ctypeslib as npct

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libmaze_poisson_ref.so")
REF_FAST_SO = os.path.join(HERE, "_ref", "libmaze_poisson_ref_fast.so")
# Source tree of the reference project (Crivella/MaZe_Poisson): MAZE_REFERENCE_ROOT, else
# the read-only checkout this build was made against.
REF_TREE = os.environ.get("MAZE_REFERENCE_ROOT", "/root/reference")


def build(ref=True):
    """Compile liboracle.so (and the reference build when its sources are present)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    if ref and os.path.isdir(os.path.join(REF_TREE, "library", "src")):
        subprocess.run(["make", "-s", "-C", HERE, "ref", f"REF_ROOT={REF_TREE}"], check=True)


def oracle_path():
    if not os.path.exists(ORACLE_SO) or (
            os.path.getmtime(ORACLE_SO) < os.path.getmtime(os.path.join(HERE, "oracle.c"))):
        build(ref=False)
    return ORACLE_SO


_f = npct.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_i64 = npct.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")
_i32 = npct.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_c = ctypes
KERNELS = {
    "orc_laplace": (None, [_f, _f, _c.c_int]),
    "orc_conj_grad": (_c.c_int, [_f, _f, _f, _c.c_double, _c.c_int]),
    "orc_smooth_rbgs": (None, [_f, _f, _c.c_int, _c.c_int]),
    "orc_restrict27": (None, [_f, _f, _c.c_int]),
    "orc_prolong_trilinear": (None, [_f, _f, _c.c_int]),
    "orc_cg_coarse": (_c.c_int, [_f, _f, _c.c_int, _c.c_int, _c.c_double]),
    "orc_mg_apply": (None, [_f, _f, _c.c_int, _c.c_int]),
    "orc_cic_neighbors": (None, [_f, _c.c_int, _c.c_int, _c.c_double, _i64]),
    "orc_spread_cic": (_c.c_double, [_f, _f, _i64, _c.c_int, _c.c_int, _c.c_double, _f]),
    "orc_force_fd": (_c.c_double, [_f, _i64, _f, _f, _c.c_int, _c.c_int, _c.c_double, _f]),
    "orc_spline_neighbors": (None, [_f, _c.c_int, _c.c_int, _c.c_double, _i64]),
    "orc_spread_scheme": (_c.c_double, [_f, _f, _c.c_int, _c.c_int, _c.c_double, _c.c_int, _f, _c.c_void_p]),
    "orc_force_scheme": (_c.c_double, [_f, _f, _f, _c.c_int, _c.c_int, _c.c_double, _c.c_int, _f]),
    "orc_tf_forces": (_c.c_double, [_f, _i32, _f, _c.c_int, _c.c_int, _c.c_double, _c.c_double, _f]),
    "orc_tf_table": (None, [_f, _c.c_int, _c.c_double, _f]),
    "orc_cell_list": (None, [_f, _c.c_int, _c.c_double, _c.c_int, _i32, _i32]),
    "orc_set_noise": (None, [_f, _c.c_int64]),
    "orc_update_eps_k2": (None, [_f, _f, _c.c_int, _c.c_int, _c.c_double, _c.c_double, _c.c_double,
                                 _c.c_double, _c.c_double, _f, _f, _f, _f]),
    "orc_laplace_pb": (None, [_f, _f, _f, _f, _f, _f, _c.c_int]),
    "orc_conj_grad_pb": (_c.c_int, [_f, _f, _f, _c.c_double, _c.c_int, _f, _f, _f, _f]),
    "orc_smooth_pb": (None, [_f, _f, _c.c_int, _c.c_int, _f, _f, _f, _f]),
    "orc_restrict_eps": (None, [_f, _f, _c.c_int, _c.c_int]),
    "orc_restrict_k2": (None, [_f, _f, _c.c_int]),
    "orc_cg_coarse_pb": (_c.c_int, [_f, _f, _c.c_int, _c.c_int, _c.c_double, _f, _f, _f, _f]),
    "orc_mg_pb_apply": (None, [_f, _f, _c.c_int, _c.c_int, _f, _f, _f, _f]),
    "orc_forces_pb": (None, [_f, _f, _c.c_int, _c.c_int, _c.c_double, _c.c_double, _c.c_double,
                             _c.c_double, _c.c_double, _c.c_int, _f, _f, _f, _f, _f, _f, _f, _f]),
    "orc_get_pb_grids": (None, [_f, _f, _f, _f]),
    "orc_ssor_apply": (None, [_f, _f, _c.c_int]),
    "orc_blockjacobi_apply": (None, [_f, _f, _c.c_int]),
    "orc_blockjacobi_inverse": (None, [_f]),
}


def load_kernels(path=None):
    """ctypes handle of the oracle with its orc_* kernels typed."""
    lib = ctypes.CDLL(path or oracle_path(), mode=ctypes.RTLD_LOCAL)
    for name, (res, args) in KERNELS.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib
