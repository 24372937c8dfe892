"""CPU check of the assembly's pair functions.

The Rankine and wave functions that the assembly kernels call per pair of
panels, compiled for the host (tests/host_pairs/host_pairs.cu) and applied to
every pair the way the two assembly passes do, against the oracle's influence
matrices at the GPU parity test's tolerances: 1e-12 of each row's largest entry
in deep water, 1e-10 in finite depth. Frequencies run in each case's order, so
the free-surface-panel quadrature state NQ carries over as in the reference.
This runs without a GPU; the same functions on the device are checked by the
GPU parity tests."""
import ctypes
import os
import subprocess

import numpy as np
import pytest

import gpu_cases as G
from nemoh_b200 import build as B

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(os.path.dirname(HERE), "nemoh_b200", "csrc")
SRC = os.path.join(HERE, "host_pairs", "host_pairs.cu")
LIB = os.path.join(HERE, "host_pairs", "_build", "libhost_pairs.so")
DEPS = [SRC] + [os.path.join(CSRC, f) for f in ("common.cuh", "green.cuh", "assembly.cuh", "fd_setup.cpp",
                                                "fd_setup.h")]
_d = ctypes.POINTER(ctypes.c_double)
_i = ctypes.POINTER(ctypes.c_int)


def _lib():
    if not os.path.exists(LIB) or any(os.path.getmtime(p) > os.path.getmtime(LIB) for p in DEPS):
        os.makedirs(os.path.dirname(LIB), exist_ok=True)
        subprocess.run([B.NVCC, "-std=c++17", "-O2", "-gencode", "arch=compute_100a,code=sm_100a", "-Xcompiler",
                        "-fPIC,-ffp-contract=off", "-shared", "-o", LIB, SRC, os.path.join(CSRC, "fd_setup.cpp")],
                       check=True)
    L = ctypes.CDLL(LIB)
    L.host_pairs_assemble.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, _d, _i, _d, ctypes.c_double, _d,
                                      ctypes.c_double, ctypes.c_double, ctypes.c_double, _i, _i, _d, _d, _d, _d]
    return L


CASES = G.small_cases()


@pytest.mark.parametrize("case", CASES, ids=[c.name for c in CASES])
def test_host_pair_functions_match_oracle(case):
    L = _lib()
    m = case.mesh
    n = m.npanels
    o = G.oracle_for(case)
    geo, zer = o.geometry()
    geo = np.ascontiguousarray(geo)
    _, _, apd = o.tables()
    apd = np.ascontiguousarray(apd.transpose(0, 2, 1)).ravel()
    nodes = np.ascontiguousarray(m.nodes, dtype=np.float64)
    panels = np.ascontiguousarray(m.panels, dtype=np.int32)
    p = lambda a: a.ctypes.data_as(_d)
    nq = ctypes.c_int(0)
    for w in case.omegas:
        mats = [np.zeros((n, n), dtype=np.complex128, order="F") for _ in range(4)]
        mode = ctypes.c_int()
        st = L.host_pairs_assemble(len(nodes), n, m.isym, p(nodes), panels.ctypes.data_as(_i), p(geo), zer, p(apd),
                                   case.g, case.depth, w, ctypes.byref(nq), ctypes.byref(mode),
                                   *[p(a) for a in mats])
        assert st == 0
        ref, mode_o, _ = o.assemble(w)
        assert mode.value == mode_o
        tol = 1e-10 if mode_o else 1e-12
        for a, b in zip(mats, ref):
            row = np.abs(b).max(axis=1, keepdims=True)
            err = np.abs(a - b) / row
            assert err.max() < tol, (case.name, w, err.max(), np.unravel_index(err.argmax(), err.shape))
