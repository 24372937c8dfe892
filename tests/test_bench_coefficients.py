"""bench.py's per-coefficient error table (mixed against FP64) on CPU: the
largest error over the frequencies of each excitation, added-mass and damping
coefficient, with vanishing families measured against the block maximum."""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _case():
    sys.path.insert(0, ROOT)
    from nemoh_b200 import cases as C
    return C.config_barge(n_omega=4, nx=4, ny=2, nz=2, nye=2)


def test_table_names_and_planted_error():
    sys.path.insert(0, ROOT)
    import bench
    case = _case()
    nf, nb, nr = len(case.force), len(case.betas_deg), len(case.rad)
    rng = np.random.default_rng(1)
    F64 = rng.normal(size=(nf, nb + nr, 4)) + 1j * rng.normal(size=(nf, nb + nr, 4))
    F = F64.copy()
    F[2, nb + 4, 1] += 1e-7 * abs(F64[2, nb + 4, 1].real)   # heave force, pitch radiation, real part
    t = bench.coefficient_errors(F, F64, case)
    assert t["forces"] == ["surge", "sway", "heave", "roll", "pitch", "yaw"]
    assert list(t["added_mass"]) == t["forces"] and list(t["damping"]) == t["forces"]
    assert len(t["excitation"]) == nb
    assert 0.9e-7 < t["added_mass"]["pitch"][2] < 1.1e-7
    assert t["damping"]["pitch"][2] == 0.0
    assert max(max(v) for v in t["excitation"].values()) == 0.0


def test_vanishing_family_against_block_maximum():
    sys.path.insert(0, ROOT)
    import bench
    case = _case()
    nf, nb, nr = len(case.force), len(case.betas_deg), len(case.rad)
    F64 = np.ones((nf, nb + nr, 4), dtype=complex)
    F64[1, 0, :] = 1e-14                        # sway excitation at beta = 0 vanishes by symmetry
    F = F64.copy()
    F[1, 0, :] = 3e-14                          # round-off of the other path
    t = bench.coefficient_errors(F, F64, case)
    assert t["excitation"]["beta=0"][1] < 1e-7  # 2e-14 against 1e-6 of the block maximum
