"""Build libmaze_poisson.so (the drop-in C-ABI library) for B200 with nvcc.

Compiles every CUDA source under csrc/ for sm_100a and links them into
maze_poisson_b200/libmaze_poisson.so (in-tree, so it travels with the working tree).
FP64 kernels are compiled with --fmad=false so a*b+c is rounded twice, like the
reference's C; the compute-bound pair-force kernel keeps FMA (see tf_forces.cu).

    python -m maze_poisson_b200.build [--force]
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libmaze_poisson.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
          "-Xptxas", "-warn-spills"]
# source -> extra flags
SOURCES = {
    "engine.cu": ["--fmad=false"],
    "cg_fast.cu": ["--fmad=false"],
    "particles.cu": ["--fmad=false"],
    "tf_forces.cu": ["--fmad=true"],
    "fft.cu": ["--fmad=false"],
    "facade.cu": ["--fmad=false"],
    "noalloc.cu": ["--fmad=false"],
    "mixed.cu": ["--fmad=true"],
    "pb.cu": ["--fmad=false"],
    "devmem.cu": ["--fmad=false"],
}
HEADERS = ["mzb_common.cuh", "engine.cuh", "particles.cuh", "fft.cuh", "tma.cuh", "mixed.cuh", "pb.cuh"]


def _nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.isabs(cand) and os.path.exists(cand) or not os.path.isabs(cand)):
            return cand
    return "nvcc"


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False, verbose=False):
    """Compile (if needed) and return the path of libmaze_poisson.so."""
    os.makedirs(BUILD, exist_ok=True)
    nvcc = _nvcc()
    headers = [os.path.join(CSRC, h) for h in HEADERS]
    objs = []
    for src, extra in SOURCES.items():
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src.replace(".cu", ".o"))
        objs.append(o)
        if force or _stale(o, [s] + headers + [__file__]):
            cmd = [nvcc] + ARCH + COMMON + extra + ["-c", s, "-o", o]
            if verbose:
                print(" ".join(cmd), flush=True)
            subprocess.run(cmd, check=True)
    if force or _stale(LIB, objs):
        cmd = [nvcc] + ARCH + ["-shared", "-o", LIB] + objs + ["-Xlinker", "-Bsymbolic"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
