"""Device memory exhaustion through the C-ABI is a status code, and it leaves
nothing behind: a half mesh of 76,000 panels needs 2 x 76,000^2 complex FP64
entries (185 GB) per matrix, more than the device holds, so the solve returns
ENOMEM at its first allocation, before any kernel runs on that mesh. A context
created afterwards in the same thread must solve normally: the failed
allocation's error is consumed where it is reported, not left for the next
context's launch checks (a cudaGetLastError after a launch)."""
import numpy as np
import pytest

import gpu_cases as G
import nemoh_b200 as nb
from nemoh_b200 import cases as C

pytestmark = pytest.mark.gpu


def _small_forces():
    case = C.config_cylinder(n_omega=2)
    nvel, nds, _ = G.problems(case)
    with nb.Solver(0, nb.FP64) as s:
        s.set_case(case)
        return s.solve_frequencies(case.omegas, nvel, nds)


def test_out_of_memory_is_a_status_and_later_contexts_work():
    before = _small_forces()
    big = C.Case(C.box_mesh(nx=250, ny=40, nz=200, half=True), np.array([1.0]), np.array([0.0]),
                 C.six_dofs(), C.six_dofs(), depth=0.0)
    assert big.mesh.npanels == 76000
    with nb.Solver(0, nb.FP64) as s:
        s.set_case(big)
        with pytest.raises(nb.NemohError) as ei:
            s.solve_potential(2.0 * np.pi, np.zeros(2 * big.mesh.npanels, dtype=np.complex128))
        assert ei.value.code == 21   # NEMOH_B200_ENOMEM
    after = _small_forces()
    scale = np.abs(before).max()
    assert np.abs(after - before).max() <= 1e-12 * scale
