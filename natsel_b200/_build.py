"""Build the CUDA library libnatsel_gpu.so in-tree for sm_100a.

The kernels need IEEE-exact f32 arithmetic without contraction
(--fmad=false, IEEE division and square root) so their results match the
reference solver's f32 bits.
"""
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libnatsel_gpu.so")
SOURCES = ["natsel_gpu.cu", "nsd_math.cuh", "nsd_geom.cuh", "nsd_types.cuh", "nsd_kernels.cuh", "nsd_solve.cuh",
           "nsd_ad.cuh", "nsd_adjoint.cuh", "nsd_adjoint_host.h"]

NVCC_FLAGS = [
    "-std=c++17", "-O3", "-lineinfo",
    "-gencode", "arch=compute_100a,code=sm_100a",
    "--fmad=false", "-prec-div=true", "-prec-sqrt=true", "-ftz=false",
    "-Xcompiler", "-fPIC", "-shared",
]


def nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.sep not in cand or os.path.exists(cand)):
            return cand
    return "nvcc"


def needs_build():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    include = os.path.join(HERE, "..", "include", "natsel_gpu.h")
    deps = [os.path.join(CSRC, s) for s in SOURCES] + [include]
    return any(os.path.getmtime(p) > t for p in deps if os.path.exists(p))


def build(force=False, verbose=False):
    """Compile libnatsel_gpu.so next to this file (skipped when up to date)."""
    if not force and not needs_build():
        return LIB
    cmd = [nvcc()] + NVCC_FLAGS + ["-o", LIB, os.path.join(CSRC, "natsel_gpu.cu")]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True, cwd=CSRC)
    return LIB


if __name__ == "__main__":
    build(force=True, verbose=True)
