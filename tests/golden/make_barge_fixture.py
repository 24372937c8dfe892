"""Golden values of the FP64 oracle on the full barge (the headline workload).

The barge 100 x 20 m, draft 10 m, depth 50 m, y-symmetric half mesh of 2,400
panels (nemoh_b200.cases.config_barge), 9 problems per frequency (headings
0/45/90 deg, then the 6 radiation DOFs), at two of its 40 frequencies, solved
in this order:
  * omega = 0.05 + 15 * 2.45/39 = 0.9923 rad/s: finite depth (k0 h = 5.0 < 20,
    Solver/Core/SOLVE_BEM.f90:66), which sets the NQ state
    (Solver/Core/SOLVE_BEM_FD_DIRECT.f90:99);
  * omega = 0.05 + 36 * 2.45/39 = 2.3115 rad/s: deep water (k0 h = 27.2 >= 20),
    which reads that NQ (Solver/Core/SOLVE_BEM_INFD_DIRECT.f90:78-79).

Forces come from the oracle's drop-in Solver run over the case files
(Normalvelocities.dat, Integration.dat -> results/Forces.dat, 17 digits), as
the reference's Solver executable produces them; the source strengths ZIGB and
ZIGS of every problem come from the oracle's SOLVE_POTENTIAL_* boundary, kept
at every 24th panel. The oracle needs about three minutes per frequency on one
core here, so the values are committed instead of recomputed by the tests.

Usage: python tests/golden/make_barge_fixture.py   (writes barge2400_fp64.json)
"""
import json
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

OMEGA_INDEX = (15, 36)
STRIDE = 24


def barge_case():
    from nemoh_b200 import cases as C
    case = C.config_barge(n_omega=40)
    case.omegas = case.omegas[list(OMEGA_INDEX)]
    return case


def main():
    import gpu_cases as G
    import oracle_lib as O
    from nemoh_b200 import cases as C
    case = barge_case()
    with tempfile.TemporaryDirectory() as tmp:
        F = G.oracle_forces(case, tmp)
    m = case.mesh
    o = O.Oracle(m.nodes, m.panels, m.isym, case.rho, case.g, case.depth, cache_s=True)
    nv = C.body_conditions(case)
    npb = len(case.betas_deg) + len(case.rad)
    keep = np.arange(0, m.npanels, STRIDE)
    zigb = np.zeros((len(keep), npb, len(case.omegas)), np.complex128)
    zigs = np.zeros_like(zigb)
    nexp = []
    for j in range(nv.shape[1]):
        w = case.omegas[j // npb]
        r = o.solve_problem(2 * np.pi / w, nv[:, j])
        zigb[:, j % npb, j // npb] = r["zigb"][keep]
        zigs[:, j % npb, j // npb] = r["zigs"][keep]
        if j % npb == 0:
            nexp.append(r["nexp"])
    fx = {
        "case": "config_barge(n_omega=40), omegas at indices %s, in that order" % (list(OMEGA_INDEX),),
        "omega_index": list(OMEGA_INDEX),
        "omegas": [float(w) for w in case.omegas],
        "nexp": nexp,
        "n_panels": int(m.npanels),
        "panel_stride": STRIDE,
        "forces_re": F.real.tolist(), "forces_im": F.imag.tolist(),   # (nint, 9, 2)
        "zigb_re": zigb.real.tolist(), "zigb_im": zigb.imag.tolist(),  # (panels kept, 9, 2)
        "zigs_re": zigs.real.tolist(), "zigs_im": zigs.imag.tolist(),
    }
    out = os.path.join(HERE, "barge2400_fp64.json")
    with open(out, "w") as f:
        json.dump(fx, f)
    print("wrote", out, os.path.getsize(out), "bytes")


if __name__ == "__main__":
    main()
