"""Load the reference's verification fixtures (tests/golden/verification_*.json)."""
import json
import os

import numpy as np

from nemoh_b200 import cases as C

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load(name):
    with open(os.path.join(GOLDEN, "verification_%s.json" % name)) as f:
        return json.load(f)


def case_from_fixture(fx, omegas=None):
    meshes, rad, frc = [], [], []
    for b, body in enumerate(fx["bodies"]):
        meshes.append(C.Mesh(np.array(body["nodes"]), np.array(body["panels"]), isym=body["isym"]))
        rad += [C.Dof(int(r[0]), r[1:4], r[4:7], b + 1) for r in body["rad"]]
        frc += [C.Dof(int(r[0]), r[1:4], r[4:7], b + 1) for r in body["force"]]
    mesh = C.merge_meshes(meshes) if len(meshes) > 1 else meshes[0]
    om = np.array(fx["omegas"] if omegas is None else omegas, dtype=np.float64)
    return C.Case(mesh, om, np.array(fx["betas_deg"], dtype=np.float64), rad, frc,
                  rho=fx["rho"], g=fx["g"], depth=fx["depth"])


def read_forces(path):
    return np.loadtxt(path, ndmin=2)


def radiation_coefficients(F, nbeta, nrad, n_omega):
    """Forces.dat -> added mass A[w, force, dof], damping B[w, force, dof]."""
    npb = nbeta + nrad
    A = np.zeros((n_omega, F.shape[0], nrad))
    B = np.zeros_like(A)
    for iw in range(n_omega):
        for j in range(nrad):
            col = iw * npb + nbeta + j
            A[iw, :, j] = F[:, 2 * col]
            B[iw, :, j] = F[:, 2 * col + 1]
    return A, B


def compare_cw(fx, A, B, omega_mask=None, floor=1e-2):
    """Errors of (A, B) against the fixture's CM/CA families.

    Each family (force on body fb, motion of body mb, DOF pair i,j) is scaled by
    max(family max, floor * largest family max of the same unit class), where
    the unit class is (translation|rotation of i, translation|rotation of j).
    Families that vanish by symmetry so compare against the physical size of
    the block instead of against their own round-off noise.
    Returns a list of (error, key, omega index).
    """
    cw = fx["cw"]
    nw = len(fx["omegas"])
    ucls = lambda i, j: (int(i > 3), int(j > 3))
    big = {}
    for key, fam in cw.items():
        _, _, i, j = (int(v) for v in key.split(","))
        for q in ("cm", "ca"):
            k = ucls(i, j) + (q,)
            big[k] = max(big.get(k, 0.0), fam[q + "_max"])
    out = []
    for key, fam in cw.items():
        fb, mb, i, j = (int(v) for v in key.split(","))
        fi = (fb - 1) * 6 + i - 1
        mj = (mb - 1) * 6 + j - 1
        for q, nm in (("cm", A), ("ca", B)):
            scale = max(fam[q + "_max"], floor * big[ucls(i, j) + (q,)], 1e-300)
            for iw in range(nw):
                if omega_mask is not None and not omega_mask[iw]:
                    continue
                out.append((abs(nm[iw, fi, mj] - fam[q][iw]) / scale, key + ":" + q, iw))
    return out
