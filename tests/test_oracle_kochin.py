"""Kochin function of the oracle (COMPUTE_KOCHIN.f90) against far-field energy
conservation: the radiation damping of a mode equals 4 pi rho omega k times the
integral of |H(theta)|^2 over the directions, in this normalisation
(H = 1/(4 pi) sum sigma ZS, deep water). Checked on the 300-panel cylinder at
omega = 1.05 rad/s, away from its irregular frequencies, to the mesh's
discretisation level (10%); the GPU path is compared with the oracle to 1e-9
in test_gpu_parity.py."""
import numpy as np

import gpu_cases as G
from nemoh_b200 import cases as C


def test_damping_equals_far_field_energy_flux():
    case = G.small_cases()[0]
    o = G.oracle_for(case)
    nv = C.body_conditions(case)
    nds = C.generalised_normals(case)
    npb = len(case.betas_deg) + len(case.rad)
    wi = 1
    w = case.omegas[wi]
    T = 2 * np.pi / w
    k = w * w / case.g
    th = np.linspace(0, 2 * np.pi, 361)[:-1]
    for dof in (0, 2):   # surge, heave
        r = o.solve_problem(T, nv[:, wi * npb + len(case.betas_deg) + dof])
        B = -(-(case.rho * 1j * w * r["zpb"]) @ nds[dof]).real
        H = o.kochin(T, th, r["zigb"])[:, 0]
        flux = 4 * np.pi * case.rho * w * k * np.sum(np.abs(H) ** 2) * (th[1] - th[0])
        assert abs(B / flux - 1) < 0.1, (dof, B, flux)
    # heave of an axisymmetric body radiates the same in every direction
    assert np.ptp(np.abs(H)) < 1e-9 * np.abs(H).max()
