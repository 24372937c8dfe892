"""Pin the CPU oracle against the reference's own verification results.

Nemoh's Verification/ directory holds three solver cases with reference
coefficients (added mass, damping, excitation). The oracle must reproduce
them: deep-water cases to 1e-4 of each coefficient family's magnitude
(observed ~3e-5, the single-precision level of the stored results), the
finite-depth two-body case to 2e-2 at the lower frequencies (observed
max ~8e-3, median ~1e-4; the high frequencies sit near irregular
frequencies where single and double precision runs legitimately diverge).
"""
import os

import numpy as np
import pytest

import oracle_lib
import verification as V
from nemoh_b200 import cases as C


def _run(fx, tmp_path, omegas=None):
    case = V.case_from_fixture(fx, omegas)
    C.write_case(case, str(tmp_path))
    oracle_lib.run_case(str(tmp_path))
    F = V.read_forces(os.path.join(str(tmp_path), "case", "results", "Forces.dat"))
    return case, F


@pytest.mark.parametrize("name", ["Cylinder", "NonSymmetrical"])
def test_deep_water_radiation(name, tmp_path):
    fx = V.load(name)
    case, F = _run(fx, tmp_path)
    A, B = V.radiation_coefficients(F, len(case.betas_deg), len(case.rad), len(case.omegas))
    errs = V.compare_cw(fx, A, B)
    worst = max(errs)
    assert worst[0] < 1e-4, worst
    assert np.median([e[0] for e in errs]) < 1e-5


@pytest.mark.parametrize("name", ["Cylinder", "NonSymmetrical"])
def test_deep_water_excitation(name, tmp_path):
    fx = V.load(name)
    fex = fx["fex"]
    case, F = _run(fx, tmp_path, omegas=fex["omega"])
    fk = C.froude_krylov(case)
    npb = len(case.betas_deg) + len(case.rad)
    for k, mag in enumerate(fex["mag"]):
        col = k * npb
        fdiff = F[:, 2 * col] * np.exp(1j * F[:, 2 * col + 1])
        fexc = np.abs(fdiff + fk[k, 0, :])
        mag = np.array(mag)
        scale = np.r_[[np.abs(mag[:3]).max()] * 3, [np.abs(mag[3:]).max()] * 3]
        assert np.max(np.abs(fexc - mag) / scale) < 1e-4


def test_finite_depth_two_bodies(tmp_path):
    fx = V.load("2Bodies")
    om = np.array(fx["omegas"])
    keep = om <= 1.5
    fx2 = dict(fx)
    fx2["omegas"] = list(om[keep])
    fx2["cw"] = {k: dict(v, ca=list(np.array(v["ca"])[keep]), cm=list(np.array(v["cm"])[keep]))
                 for k, v in fx["cw"].items()}
    case, F = _run(fx2, tmp_path)
    A, B = V.radiation_coefficients(F, len(case.betas_deg), len(case.rad), len(case.omegas))
    errs = V.compare_cw(fx2, A, B)
    assert max(errs)[0] < 2e-2, max(errs)
    assert np.median([e[0] for e in errs]) < 1e-3
