"""Why the influence matrices are assembled in FP64 in both precision modes.

The mixed-precision path keeps D and S in FP64 and lowers the precision of the
factorization only, recovering FP64 accuracy by refinement against the FP64
D. Lowering the precision of the matrices themselves cannot be recovered that
way: the oracle's matrices rounded entry by entry to single precision (the
best an FP32 assembly could do) and then solved exactly already miss the 1e-6
coefficient budget (per-coefficient metric of the benchmark) on a jittered
hemisphere, while an FP32 LU refined against the FP64 matrices meets it. Both
are computed here with numpy on the oracle's matrices (CPU)."""
import numpy as np
import pytest
import scipy.linalg as sla

import bench
import gpu_cases as G


def _forces(case, mats, nvel, nds, solve):
    N = case.mesh.npanels
    F = np.zeros((nds.shape[0], nvel.shape[1], nvel.shape[2]), complex)
    for w, (Dp, Dm, Sp, Sm) in enumerate(mats):
        v = nvel[:, :, w]
        if case.mesh.isym:
            pp = Sp @ solve(Dp, (v[:N] + v[N:]) / 2)
            pm = Sm @ solve(Dm, (v[:N] - v[N:]) / 2)
            z = np.concatenate([pp + pm, pp - pm])
        else:
            z = Sp @ solve(Dp, v)
        F[:, :, w] = -nds @ (case.rho * 1j * case.omegas[w] * z)
    return F


def _fp32_lu_refined(D, b, tol=1e-12, max_it=30):
    """FP32 LU (complex64) with FP64 residuals, the scheme of the mixed path."""
    lu = sla.lu_factor(D.astype(np.complex64))
    x = sla.lu_solve(lu, b.astype(np.complex64)).astype(np.complex128)
    bn = np.abs(b).max(axis=0)
    for _ in range(max_it):
        r = b - D @ x
        if (np.abs(r).max(axis=0) <= tol * bn).all():
            break
        x += sla.lu_solve(lu, r.astype(np.complex64)).astype(np.complex128)
    return x


@pytest.fixture(scope="module")
def hemisphere():
    case = [c for c in G.small_cases() if c.name == "sphere_deep"][0]
    o = G.oracle_for(case)
    mats = [o.assemble(w)[0] for w in case.omegas]
    nvel, nds, _ = G.problems(case)
    F64 = _forces(case, mats, nvel, nds, np.linalg.solve)
    return case, mats, nvel, nds, F64


def test_fp32_matrices_miss_the_budget(hemisphere):
    case, mats, nvel, nds, F64 = hemisphere
    r32 = [tuple(m.astype(np.complex64).astype(np.complex128) for m in ms) for ms in mats]
    err, _ = bench.rel_err_families(_forces(case, r32, nvel, nds, np.linalg.solve), F64, len(case.betas_deg))
    assert err > 1e-5, err   # observed 4.5e-5


def test_fp32_factors_refined_against_fp64_matrices_meet_it(hemisphere):
    case, mats, nvel, nds, F64 = hemisphere
    err, _ = bench.rel_err_families(_forces(case, mats, nvel, nds, _fp32_lu_refined), F64, len(case.betas_deg))
    assert err < 1e-8, err


def _near_field(o, case):
    """Pairs (I, J) whose Rankine integral the reference evaluates exactly:
    RO <= 7 TDIS(J) for one of the images the pair is summed over (direct,
    free-surface image, y-mirrors; COMPUTE_GREEN_INFD.f90:80-98)."""
    geo, _ = o.geometry()
    XG, YG, ZG, T = geo[3], geo[4], geo[5], geo[7]
    ro = []
    for sy in ((1.0, -1.0) if case.mesh.isym else (1.0,)):
        for zj in (ZG, -ZG):
            ro.append(np.sqrt((XG[:, None] - XG[None, :]) ** 2 + (YG[:, None] - sy * YG[None, :]) ** 2 +
                              (ZG[:, None] - zj[None, :]) ** 2))
    return np.min(ro, axis=0) <= 7.0 * T[None, :]


def test_fp32_far_field_split_misses_the_budget(hemisphere):
    """The split of near-field pairs in FP64 and far-field pairs in FP32, at
    its most favourable: near-field entries exact, far-field entries the FP64
    values rounded to single precision (the least error an FP32 evaluation of
    them can have). Solved exactly, it still misses 1e-6 on the jittered
    hemisphere (observed 1.8e-5; 76% of its pairs are near field)."""
    case, mats, nvel, nds, F64 = hemisphere
    o = G.oracle_for(case)
    near = _near_field(o, case)
    split = [tuple(np.where(near, m, m.astype(np.complex64).astype(np.complex128)) for m in ms) for ms in mats]
    err, _ = bench.rel_err_families(_forces(case, split, nvel, nds, np.linalg.solve), F64, len(case.betas_deg))
    assert err > 1e-6, err
