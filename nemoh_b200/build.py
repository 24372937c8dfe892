"""Build libnemoh_b200.so (sm_100a) and the drop-in Solver and post-processor executables in-tree.

    python -m nemoh_b200.build        # or nemoh_b200.build.build()

nvcc cross-compiles for sm_100a without a GPU. Outputs go to
nemoh_b200/_build/ next to the sources, so the built library travels with the
source tree.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "_build")
LIB = os.path.join(OUT, "libnemoh_b200.so")
DRIVER = os.path.join(OUT, "nemoh_solver_b200")
POSTPROC = os.path.join(OUT, "nemoh_postproc_b200")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# host code: no FMA contraction, same as the reference's -O2 x86-64 build
HOSTFLAGS = ["-Xcompiler", "-fPIC,-ffp-contract=off"]
COMMON = ["-std=c++17", "-O3", "-lineinfo"] + ARCH + HOSTFLAGS


def _sources(names):
    return [os.path.join(CSRC, n) for n in names]


LIB_SRC = ["api.cu", "fd_setup.cpp"]
DEPS = ["api.cu", "fd_setup.cpp", "fd_setup.h", "common.cuh", "green.cuh", "assembly.cuh", "linalg.cuh",
        "mixed.cuh", "tc_gemm.cuh", "tune.cuh", "kochin.cuh", "preproc.cuh", "freesurface.cuh", "postproc.cuh", "case_io.h", "driver.cpp", "postproc.cpp"]


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    hdr = os.path.join(os.path.dirname(HERE), "include", "nemoh_b200.h")
    return any(os.path.getmtime(p) > t for p in _sources(deps) + [hdr] if os.path.exists(p))


def build(force=False, verbose=False):
    os.makedirs(OUT, exist_ok=True)
    if force or _stale(LIB, DEPS):
        # static CUDA runtime: independent of the runtime version other libraries
        # (e.g. torch) load into the same process
        cmd = [NVCC] + COMMON + ["-shared", "-cudart", "static", "-o", LIB] + _sources(LIB_SRC)
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    for exe, src in ((DRIVER, "driver.cpp"), (POSTPROC, "postproc.cpp")):
        path = os.path.join(CSRC, src)
        if force or _stale(exe, [src, "case_io.h"]) or os.path.getmtime(exe) < os.path.getmtime(LIB):
            cmd = ["g++", "-std=c++17", "-O2", "-ffp-contract=off", "-Wall", "-o", exe, path,
                   "-I" + os.path.join(os.path.dirname(HERE), "include"),
                   "-L" + OUT, "-lnemoh_b200", "-Wl,-rpath,$ORIGIN"]
            if verbose:
                print(" ".join(cmd))
            subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
