"""B200-native drop-in for the per-step MD hot path of MaZe_Poisson.

The product is libmaze_poisson.so (built from csrc/ by build.py for sm_100a): a C-ABI
library exporting the reference's symbols (include/maze_poisson.h) whose every compute
step runs as hand-written CUDA on the GPU. This package adds the ctypes binding
(c_api.py), a synthetic molten-salt generator (systems.py) and an MD driver mirroring
the reference's SolverMD call sequence (md.py).

There is no CPU fallback: importing the binding without the built library raises.
"""
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_NAME = "libmaze_poisson.so"


def library_path(require=False):
    """Path of the in-tree libmaze_poisson.so; raise if `require` and it is missing."""
    path = os.path.join(_HERE, LIB_NAME)
    if require and not os.path.exists(path):
        raise RuntimeError(
            f"{path} is missing: build it with `python -m maze_poisson_b200.build` "
            "(this package has no CPU fallback)")
    return path
