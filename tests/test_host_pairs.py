"""CPU check of the kernels' pair functions.

The Rankine and wave functions that the assembly kernels call per pair of
panels, compiled for the host (tests/host_pairs/host_pairs.cu) and applied to
every pair the way the two assembly passes do, against the oracle's influence
matrices at the GPU parity test's tolerances: 1e-12 of each row's largest entry
in deep water, 1e-10 in finite depth. Frequencies run in each case's order, so
the free-surface-panel quadrature state NQ carries over as in the reference.
Likewise the field-point Green functions of the free-surface kernel against the
oracle's elevation for the same source strengths (1e-9 of each problem's
largest |ETA|), and the Kochin kernel's panel integrals against the oracle's
Kochin function (1e-9 of the largest |H|), and the body-conditions kernel's
panel quantities and radiation conditions against the pre-processor
restatement (1e-12); and the wave pass's enumeration of upper-triangle tiles.
This runs without a GPU; the same functions on the device are
checked by the GPU parity tests."""
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
DEPS = [SRC] + [os.path.join(CSRC, f) for f in ("common.cuh", "green.cuh", "assembly.cuh", "freesurface.cuh",
                                                "kochin.cuh", "preproc.cuh", "fd_setup.cpp", "fd_setup.h")]
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
    L.host_pairs_free_surface.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, _d, _i, _d, ctypes.c_double, _d,
                                          ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                          ctypes.c_int, _d, ctypes.c_int, _d, _d, _d]
    L.host_pairs_kochin.argtypes = [ctypes.c_int, ctypes.c_int, _d, _i, _d, ctypes.c_double, ctypes.c_double,
                                    ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_int, _d,
                                    ctypes.c_int, _d, _d, _d]
    L.host_pairs_preproc.argtypes = [ctypes.c_int, _d, _i, ctypes.c_int, _i, _d, _d, _d, _d]
    L.host_pairs_preproc.restype = None
    L.host_pairs_tri_tile_misses.argtypes = [ctypes.c_int]
    L.host_pairs_tri_tile_misses.restype = ctypes.c_longlong
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


def _fs_points(case):
    """A polar grid on z = 0 from just outside the waterline (tabulated wave
    term) to 30 body radii (asymptotic form)."""
    nodes = case.mesh.nodes
    r0 = np.hypot(nodes[:, 0], nodes[:, 1]).max()
    R, TH = np.meshgrid(r0 * np.array([1.15, 1.6, 3.0, 8.0, 30.0]), np.linspace(0.0, 2.0 * np.pi, 7)[:-1] + 0.1)
    return np.ascontiguousarray(np.stack([(R * np.cos(TH)).ravel(), (R * np.sin(TH)).ravel()], axis=1))


@pytest.mark.parametrize("case", CASES, ids=[c.name for c in CASES])
def test_host_free_surface_functions_match_oracle(case):
    from nemoh_b200 import cases as C
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
    nv = C.body_conditions(case)
    npb = len(case.betas_deg) + len(case.rad)
    xy = _fs_points(case)
    w_idx = len(case.omegas) - 1
    T = 2 * np.pi / case.omegas[w_idx]
    cols = [w_idx * npb, w_idx * npb + npb - 1]   # the first heading and the last DOF
    res = [o.solve_problem(T, nv[:, j]) for j in cols]
    zigb = np.asfortranarray(np.stack([r["zigb"] for r in res], axis=1))
    zigs = np.asfortranarray(np.stack([r["zigs"] for r in res], axis=1))
    eta = np.zeros((len(xy), len(cols)), dtype=np.complex128, order="F")
    st = L.host_pairs_free_surface(len(nodes), n, m.isym, p(nodes), panels.ctypes.data_as(_i), p(geo), zer, p(apd),
                                   case.g, case.depth, T, o.nq, len(xy), p(xy), len(cols), p(zigb), p(zigs), p(eta))
    assert st == 0
    eo = o.free_surface(T, xy, zigb, zigs if m.isym else None)
    scale = np.abs(eo).max(axis=0)
    assert np.all(scale > 0)
    err = (np.abs(eta - eo) / scale).max()
    assert err < 1e-9, (case.name, err)


@pytest.mark.parametrize("case", CASES, ids=[c.name for c in CASES])
def test_host_kochin_functions_match_oracle(case):
    from nemoh_b200 import cases as C
    L = _lib()
    m = case.mesh
    n = m.npanels
    o = G.oracle_for(case)
    geo, _ = o.geometry()
    geo = np.ascontiguousarray(geo)
    nodes = np.ascontiguousarray(m.nodes, dtype=np.float64)
    panels = np.ascontiguousarray(m.panels, dtype=np.int32)
    p = lambda a: a.ctypes.data_as(_d)
    nv = C.body_conditions(case)
    npb = len(case.betas_deg) + len(case.rad)
    theta = np.linspace(0.0, 2.0 * np.pi, 37)
    xeff, yeff = 1.5, -0.7
    for w_idx in (0, len(case.omegas) - 1):
        T = 2 * np.pi / case.omegas[w_idx]
        cols = list(range(w_idx * npb, (w_idx + 1) * npb))
        res = [o.solve_problem(T, nv[:, j]) for j in cols]
        zigb = np.asfortranarray(np.stack([r["zigb"] for r in res], axis=1))
        zigs = np.asfortranarray(np.stack([r["zigs"] for r in res], axis=1))
        H = np.zeros((len(theta), len(cols)), dtype=np.complex128, order="F")
        st = L.host_pairs_kochin(n, m.isym, p(nodes), panels.ctypes.data_as(_i), p(geo), case.g, case.depth, T,
                                 xeff, yeff, len(theta), p(theta), len(cols), p(zigb), p(zigs), p(H))
        assert st == 0
        Ho = o.kochin(T, theta, zigb, zigs if m.isym else None, xeff, 0.0 if m.isym else yeff)
        err = np.abs(H - Ho).max() / np.abs(Ho).max()
        assert err < 1e-9, (case.name, w_idx, err)


@pytest.mark.parametrize("case", CASES, ids=[c.name for c in CASES])
def test_host_preprocessor_functions_match_restatement(case):
    from nemoh_b200 import cases as C
    L = _lib()
    m = case.mesh
    n = m.npanels
    nodes = np.ascontiguousarray(m.nodes, dtype=np.float64)
    panels = np.ascontiguousarray(m.panels, dtype=np.int32)
    p = lambda a: a.ctypes.data_as(_d)
    dofs = case.rad
    kind = np.array([d.icase for d in dofs], dtype=np.int32)
    dr = np.ascontiguousarray([d.direction for d in dofs], dtype=np.float64)
    ax = np.ascontiguousarray([d.axis for d in dofs], dtype=np.float64)
    panel = np.zeros((7, n))
    rad = np.zeros((len(dofs), n))
    L.host_pairs_preproc(n, p(nodes), panels.ctypes.data_as(_i), len(dofs), kind.ctypes.data_as(_i), p(dr), p(ax),
                         p(panel), p(rad))
    xm, nrm, a = C.panel_quantities(m)
    for got, ref in ((panel[0:3].T, xm), (panel[3:6].T, nrm), (panel[6], a)):
        assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max()
    for d, dof in enumerate(dofs):
        ref = C._dof_vector(m, xm, nrm, a, dof, False)[:n]
        assert np.abs(rad[d] - ref).max() <= 1e-12 * max(np.abs(ref).max(), 1.0), (case.name, d)


def test_wave_pass_takes_every_upper_triangle_tile_once():
    """Block t of the wave pass maps to tile (a, b), a <= b, of the T x T grid
    of 16 x 16 tiles: every tile exactly once, for every grid up to 8,000
    panels (T = 500) and the orders of the benchmark and tests."""
    L = _lib()
    for T in list(range(1, 201)) + [250, 300, 499, 500, 501]:
        assert L.host_pairs_tri_tile_misses(T) == 0, T
