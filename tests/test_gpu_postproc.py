"""GPU: the post-processor's impulse response functions (nemoh_b200_irf) and
the drop-in post-processor executable against the oracle's restatement of
postProcessor/Main.f90. IRF tolerance: 1e-12 of the largest |K| and of the
largest |A_inf| (CUDA's and the host's cos/sin differ in the last place)."""
import dataclasses
import os
import shutil
import subprocess

import numpy as np
import pytest

import gpu_cases as G
import nemoh_b200 as nb
import oracle_lib as O
from nemoh_b200 import build as B
from nemoh_b200 import cases as C

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.parametrize("shape", [(40, 6, 6), (7, 3, 20), (150, 12, 12)])
def test_irf_matches_oracle(shape):
    B.build()
    nw, nrad, nint = shape
    rng = np.random.default_rng(nw)
    w = np.sort(rng.uniform(0.05, 3.0, nw))
    damping = rng.standard_normal(shape) * np.exp(-w)[:, None, None]
    added = rng.standard_normal(shape) + 2.0
    with nb.Solver(0, nb.FP64) as s:
        for ntime, dt in ((100, 0.1), (1, 0.5), (0, 0.1)):
            K, ainf = s.irf(w, damping, added, ntime, dt)
            Ko, ao = O.irf(w, damping, added, ntime, dt)
            if ntime:
                assert np.abs(K - Ko).max() <= 1e-12 * np.abs(Ko).max()
            assert np.abs(ainf - ao).max() <= 1e-12 * np.abs(ao).max()


def test_dropin_postprocessor_matches_oracle(tmp_path):
    """Both post-processors on the same Solver results (the oracle's run of a
    finite-depth barge with three headings and IRF on): every file identical
    except IRF.tec, whose values agree within 1e-12 of the largest."""
    B.build()
    case = dataclasses.replace(G.small_cases()[1], irf=(0.1, 8.0), betas_deg=np.array([0.0, 30.0, 90.0]))
    ref = str(tmp_path / "ref")
    C.write_case(case, ref)
    O.run_case(ref)
    gpu = str(tmp_path / "gpu")
    shutil.copytree(ref, gpu)
    O.postproc(ref)
    exe = os.path.join(ROOT, "nemoh_b200", "_build", "nemoh_postproc_b200")
    subprocess.run([exe, gpu], check=True)
    rr, rg = os.path.join(ref, "case", "results"), os.path.join(gpu, "case", "results")
    for name in ("RadiationCoefficients.tec", "DiffractionForce.tec", "ExcitationForce.tec", "CA.dat", "CM.dat",
                 "Fe.dat"):
        assert open(os.path.join(rr, name), "rb").read() == open(os.path.join(rg, name), "rb").read(), name
    a = open(os.path.join(rr, "IRF.tec")).read().split("\n")
    b = open(os.path.join(rg, "IRF.tec")).read().split("\n")
    assert len(a) == len(b) == 2 + len(case.force) + len(case.rad) * (80 + 1)
    num = lambda L: np.array([[float(v) for v in l.split()] for l in L if l and l[0] == " " and "VARIABLES" not in l])
    na, nb_ = num(a), num(b)
    assert [l for l in a if not l.startswith(" ")] == [l for l in b if not l.startswith(" ")]
    assert np.array_equal(na[:, 0], nb_[:, 0])
    assert np.abs(na - nb_).max() <= 1e-12 * np.abs(na[:, 1:]).max()
