"""FP64 parity at the sizes of the benchmark workloads, per coefficient.

* The barge of the headline workload (2,400-panel y-symmetric half mesh,
  depth 50 m, 9 problems) at one finite-depth and one deep-water frequency, in
  that order (the deep-water solve reads the NQ state the finite-depth one
  left, Solver/Core/SOLVE_BEM_INFD_DIRECT.f90:78-79), against the committed
  oracle values (tests/golden/barge2400_fp64.json, made by
  tests/golden/make_barge_fixture.py; the oracle takes minutes per frequency at
  this order): forces per coefficient, and the source strengths ZIGB/ZIGS of
  the reference boundary (nemoh_b200_solve_problem) on every 24th panel.
* The 300-panel deep-water cylinder at all 10 of its frequencies against the
  oracle run here.

Coefficient metric: |x - x_oracle| / max(|x_oracle|, 1e-6 * family max), a
family being one force component and one problem over the frequencies of the
case, with families that vanish by symmetry measured against 1e-6 of their
kind's largest coefficient (gpu_cases.coef_err).
"""
import json
import os

import numpy as np
import pytest

import gpu_cases as G
import nemoh_b200 as nb
from nemoh_b200 import build as B
from nemoh_b200 import cases as C

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
COEF_TOL = G.PARITY_TOL
SIGMA_TOL = 1e-10


def _fixture():
    with open(os.path.join(HERE, "golden", "barge2400_fp64.json")) as f:
        fx = json.load(f)
    cplx = lambda k: np.array(fx[k + "_re"]) + 1j * np.array(fx[k + "_im"])
    return fx, cplx("forces"), cplx("zigb"), cplx("zigs")


def _barge():
    case = C.config_barge(n_omega=40)
    fx, _, _, _ = _fixture()
    case.omegas = case.omegas[fx["omega_index"]]
    assert np.array_equal(case.omegas, np.array(fx["omegas"]))
    return case


@pytest.fixture(scope="module")
def solver():
    B.build()
    s = nb.Solver(0, nb.FP64)
    yield s
    s.close()


def test_barge_2400_forces_per_coefficient(solver):
    fx, Fo, _, _ = _fixture()
    case = _barge()
    solver.set_case(case)
    nvel, nds, npb = G.problems(case)
    F = solver.solve_frequencies(case.omegas, nvel, nds)
    err = G.parity_err(F, Fo, len(case.betas_deg))
    assert err < COEF_TOL, err


def test_barge_2400_source_strengths(solver):
    fx, _, zb, zs = _fixture()
    case = _barge()
    solver.set_case(case)
    nv = C.body_conditions(case)
    npb = len(case.betas_deg) + len(case.rad)
    keep = np.arange(0, case.mesh.npanels, fx["panel_stride"])
    for j in range(nv.shape[1]):
        w, p = j // npb, j % npb
        g = solver.solve_potential(2 * np.pi / case.omegas[w], nv[:, j])
        if p == 0:
            assert g["nexp"] == fx["nexp"][w]
        for got, ref in ((g["zigb"][keep], zb[:, p, w]), (g["zigs"][keep], zs[:, p, w])):
            assert np.abs(got - ref).max() <= SIGMA_TOL * np.abs(ref).max(), (w, p)


def test_cylinder_all_ten_frequencies_per_coefficient(solver, tmp_path):
    case = C.config_cylinder(n_omega=10)
    solver.set_case(case)
    nvel, nds, npb = G.problems(case)
    F = solver.solve_frequencies(case.omegas, nvel, nds)
    Fo = G.oracle_forces(case, str(tmp_path))
    err = G.parity_err(F, Fo, len(case.betas_deg))
    assert err < COEF_TOL, err
