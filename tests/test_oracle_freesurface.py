"""Free-surface elevation of the oracle (COMPUTE_POTENTIAL_DOMAIN.f90 at z = 0,
ETA = i W/G PHI as SOLVE_BEM.f90:104-109 writes it) against the far field that
the Kochin function describes: at k R >> 1 the radiated wave is
ETA(R, theta) ~ A H(theta) exp(i k R) / sqrt(R) with one constant A for every
direction. Checked on a deep-water barge (not axisymmetric, so H varies with
theta: surge has a node across the barge) for surge and heave at k a = 1.3.
The two sums treat a panel differently (the field sums each panel at its
centroid), so they agree to the mesh's discretisation level: 0.2% of max |H|
on this mesh, falling to 0.05% with panels half the size, and the same at
k R = 4e3 and 4e4."""
import numpy as np

import gpu_cases as G
from nemoh_b200 import cases as C


def test_far_field_elevation_follows_kochin_function():
    case = C.config_barge(n_omega=1, nx=8, ny=3, nz=3, nye=3)
    case.depth = 0.0
    o = G.oracle_for(case)
    nv = C.body_conditions(case)
    w = 0.5
    case.omegas = np.array([w])
    T = 2 * np.pi / w
    k = w * w / case.g
    th = np.linspace(0.0, np.pi, 7) + 0.05
    R = 4000.0 / k
    for dof in (0, 2):   # surge, heave
        r = o.solve_problem(T, nv[:, len(case.betas_deg) + dof])
        H = o.kochin(T, th, r["zigb"], r["zigs"])[:, 0]
        xy = np.stack([R * np.cos(th), R * np.sin(th)], axis=1)
        eta = o.free_surface(T, xy, r["zigb"], r["zigs"])[:, 0]
        a = np.vdot(H, eta) / np.vdot(H, H)
        assert np.abs(eta / a - H).max() < 1e-2 * np.abs(H).max(), dof
        if dof == 0:
            assert np.abs(H).min() < 0.1 * np.abs(H).max()
        # cylindrical spreading: |ETA| sqrt(R) is the same at R and 4 R
        far = o.free_surface(T, 4 * xy, r["zigb"], r["zigs"])[:, 0]
        assert np.abs(np.abs(far) * 2 / np.abs(eta) - 1).max() < 1e-3, dof
