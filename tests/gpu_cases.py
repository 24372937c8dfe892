"""Small cases and helpers shared by the GPU parity tests."""
import math
import os

import numpy as np

import oracle_lib as O
from nemoh_b200 import cases as C


def small_cases():
    """(name, Case) covering deep/finite depth, with and without symmetry."""
    cyl = C.config_cylinder(n_omega=3)
    cyl.name = "cylinder300_deep"
    barge = C.config_barge(n_omega=3, nx=10, ny=4, nz=4, nye=4)
    barge.name = "barge_half_fd50"
    half_cyl = C.Case(C.cylinder_mesh(4.0, 6.0, 16, 6, 3, 8, half=True), np.array([0.4, 1.1, 1.9]),
                      np.array([30.0]), C.six_dofs((0, 0, -2.0)), C.six_dofs((0, 0, -2.0)), depth=15.0)
    half_cyl.name = "half_cylinder_fd15"
    sph = C.Case(C.hemisphere_mesh(3.0, 8, 16, jitter=0.2, rng=np.random.default_rng(7)), np.array([0.5, 1.5]),
                 np.array([0.0, 60.0]), C.six_dofs(), C.six_dofs(), depth=0.0)
    sph.name = "sphere_deep"
    return [cyl, barge, half_cyl, sph]


def oracle_for(case, cache_s=True):
    m = case.mesh
    return O.Oracle(m.nodes, m.panels, m.isym, case.rho, case.g, case.depth, cache_s=cache_s)


def problems(case):
    """(nvel (2^s N, npb, nw), nds, omega per problem, switch_type per problem)."""
    nv = C.body_conditions(case)
    nb_, nr = len(case.betas_deg), len(case.rad)
    npb = nb_ + nr
    nw = len(case.omegas)
    nvel = nv.reshape(nv.shape[0], nw, npb).transpose(0, 2, 1)
    nds = C.generalised_normals(case)
    return np.asfortranarray(nvel), nds, npb


def oracle_forces(case, tmpdir):
    C.write_case(case, tmpdir)
    O.run_case(tmpdir)
    F = np.loadtxt(os.path.join(tmpdir, "case", "results", "Forces.dat"), ndmin=2)
    return decode_forces(case, F)


def decode_forces(case, F):
    """Forces.dat rows -> complex force (nint, npb, nw) (NEMOH.f90:152-166 inverted)."""
    nb_, nr = len(case.betas_deg), len(case.rad)
    npb = nb_ + nr
    nw = len(case.omegas)
    out = np.zeros((F.shape[0], npb, nw), dtype=np.complex128)
    for w in range(nw):
        for p in range(npb):
            j = w * npb + p
            a, b = F[:, 2 * j], F[:, 2 * j + 1]
            if p < nb_:
                out[:, p, w] = a * np.exp(1j * b)
            else:
                out[:, p, w] = -b + 1j * a * case.omegas[w]
    return out


def coef_err(a, b, nbeta, floor=1e-6, per_coef=False, vanish_floor=None):
    """Per-coefficient error of forces a against b, both (nint, nprob, nw):
    |a - b| / max(|b|, floor * family max), a family being one force component
    and one problem over all frequencies (force(i, p) over omega); the first
    nbeta problems are diffraction, the rest radiation. A family whose largest
    value is at most 1e-9 of the largest coefficient of its kind vanishes by the
    body's symmetry (both sides hold round-off there) and is measured against
    `vanish_floor` (default `floor`) times that kind maximum. Returns the
    maximum (or the array)."""
    mag = np.abs(b)
    fam = mag.max(axis=2, keepdims=True)
    kind = np.empty_like(fam)
    kind[:, :nbeta] = mag[:, :nbeta].max() if nbeta else 0.0
    kind[:, nbeta:] = mag[:, nbeta:].max() if nbeta < mag.shape[1] else 0.0
    vf = floor if vanish_floor is None else vanish_floor
    den = np.where(fam <= 1e-9 * kind, vf * kind, np.maximum(mag, floor * fam))
    err = np.abs(a - b) / np.maximum(den, 1e-300)
    return err if per_coef else float(err.max())


PARITY_TOL = 1e-9


def parity_err(a, b, nbeta):
    """The FP64 parity metric: coef_err per coefficient with the benchmark's
    floor of 1e-6 of the family maximum; families that vanish by symmetry hold
    only round-off on both sides and are measured against 1e-3 of their kind's
    largest coefficient, so that PARITY_TOL bounds their absolute difference
    by 1e-12 of that maximum."""
    return coef_err(a, b, nbeta, floor=1e-6, vanish_floor=1e-3)


def rel_err(a, b):
    """max |a-b| / max|b| per integration case (row), maximised over rows."""
    num = np.abs(a - b).reshape(a.shape[0], -1).max(axis=1)
    den = np.abs(b).reshape(b.shape[0], -1).max(axis=1)
    return float(np.max(num / np.maximum(den, 1e-300)))
