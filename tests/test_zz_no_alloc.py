"""nemoh_b200_factor_solve_device_noalloc through the C-ABI.

The entry point factors and solves device-resident systems with its scratch
in a static device array and allocates nothing. Its solutions are checked
against the context path's source strengths (nemoh_b200_solve_problem, ZIGB
and ZIGS) on the context's own influence matrices (nemoh_b200_assemble), for
two calls in a row of different sizes that share the scratch, within the
source-strength tolerance of the parity tests (1e-10). The second call must
leave the device's free memory unchanged.

The file name makes pytest collect it last; it passes alone in a fresh
process and after the other tests.
"""
import ctypes

import numpy as np
import pytest

import gpu_cases as G
import nemoh_b200 as nb
from nemoh_b200 import build as B
from nemoh_b200 import cases as C

pytestmark = pytest.mark.gpu

TOL = 1e-10
ECAPACITY = 23


def _entry():
    L = nb.load_library()
    f = L.nemoh_b200_factor_solve_device_noalloc
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                  ctypes.c_void_p, ctypes.c_char_p, ctypes.c_int]
    return f


def _reference(case, ncols):
    """Influence matrices and ZIGB/ZIGS of the context path at the first frequency."""
    omega = float(case.omegas[0])
    nv = C.body_conditions(case)[:, :ncols]
    m = case.mesh
    with nb.Solver(0, nb.FP64) as s:
        s.set_mesh(m.nodes, m.panels, m.isym, case.rho, case.g, case.depth)
        (dp, dm, _, _), _ = s.assemble(omega)
        refs = [s.solve_potential(2.0 * np.pi / omega, nv[:, p]) for p in range(ncols)]
    n = m.npanels
    mats = [dp, dm] if m.isym else [dp]
    a = np.concatenate([x.ravel(order="F") for x in mats])
    if m.isym:
        b = np.stack([np.stack([(nv[:n, p] + sgn * nv[n:, p]) * 0.5 for p in range(ncols)]) for sgn in (1.0, -1.0)])
    else:
        b = nv[None, :n, :].transpose(0, 2, 1)
    return a, np.ascontiguousarray(b), refs


def _rel(x, y):
    return float(np.abs(x - y).max() / max(np.abs(y).max(), 1e-300))


def _check(case, x, refs):
    n = case.mesh.npanels
    for p, r in enumerate(refs):
        if case.mesh.isym:
            zigb, zigs = x[0, p] + x[1, p], x[0, p] - x[1, p]
            assert _rel(zigb, r["zigb"]) < TOL and _rel(zigs, r["zigs"]) < TOL
        else:
            assert x.shape[2] == n
            assert _rel(x[0, p], r["zigb"]) < TOL


def test_noalloc_factor_solve_matches_context_path():
    import torch

    B.build()
    f = _entry()
    cases = {c.name: c for c in G.small_cases()}
    first, second = cases["cylinder300_deep"], cases["barge_half_fd50"]
    a1, b1, r1 = _reference(first, 1)
    a2, b2, r2 = _reference(second, 3)
    dev = torch.device("cuda", 0)
    # device buffers are made by the test; the entry point only uses them
    A1, X1 = torch.from_numpy(a1).to(dev), torch.from_numpy(b1).to(dev)
    A2, X2 = torch.from_numpy(a2).to(dev), torch.from_numpy(b2).to(dev)
    stream = torch.cuda.current_stream(dev)
    msg = ctypes.create_string_buffer(512)
    torch.cuda.synchronize(dev)

    st = f(0, first.mesh.npanels, b1.shape[0], A1.data_ptr(), b1.shape[1], X1.data_ptr(), stream.cuda_stream, msg,
           512)
    assert st == 0, msg.value.decode()
    _check(first, X1.cpu().numpy(), r1)

    torch.cuda.synchronize(dev)
    free0, _ = torch.cuda.mem_get_info(dev)
    st = f(0, second.mesh.npanels, b2.shape[0], A2.data_ptr(), b2.shape[1], X2.data_ptr(), stream.cuda_stream, msg,
           512)
    assert st == 0, msg.value.decode()
    torch.cuda.synchronize(dev)
    free1, _ = torch.cuda.mem_get_info(dev)
    assert free1 == free0
    _check(second, X2.cpu().numpy(), r2)


def test_noalloc_rejects_sizes_beyond_scratch():
    B.build()
    f = _entry()
    msg = ctypes.create_string_buffer(512)
    # n = 4096, two systems, 16 right-hand sides: about 18 MiB of scratch; the
    # size is rejected before any buffer is touched, so aligned dummy addresses do
    st = f(0, 4096, 2, 256, 16, 512, None, msg, 512)
    assert st == ECAPACITY
    assert b"exceeds the fixed" in msg.value


def test_noalloc_refuses_host_buffers():
    """Host memory handed in as device memory is a status code, not a fault:
    the pointers are checked before any kernel is launched."""
    B.build()
    f = _entry()
    msg = ctypes.create_string_buffer(512)
    a = np.zeros(2 * 8 * 8, dtype=np.float64)
    x = np.zeros(2 * 8, dtype=np.float64)
    st = f(0, 8, 1, a.ctypes.data, 1, x.ctypes.data, None, msg, 512)
    assert st == 1, (st, msg.value)   # NEMOH_B200_EINVAL
    assert b"host memory" in msg.value
    assert not a.any() and not x.any()
