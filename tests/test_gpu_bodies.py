"""Cross-body (ragged) batches through the C-ABI: nemoh_b200_add_body and
nemoh_b200_solve_bodies against the single-body path.

Items of bodies with different panel counts (deep and finite depth, with and
without y-symmetry) and frequencies, in a shuffled order with repeated bodies,
are solved in one call; every item's forces must equal those of
nemoh_b200_solve_frequencies on that body alone (itself checked against the
oracle in test_gpu_parity.py) within 1e-12 of the item's largest force in
FP64 (the mat-vec sums by atomics, so the last bits may differ), and in mixed
precision within 1e-10 of the single-body mixed result and 1e-6 (per
coefficient) of FP64. A device-memory budget small enough to split the call
into several batches gives the same results.
"""
import os

import numpy as np
import pytest

import gpu_cases as G
import nemoh_b200 as nb
from nemoh_b200 import build as B
from nemoh_b200 import cases as C

pytestmark = pytest.mark.gpu


def _bodies():
    out = [c for c in G.small_cases()]
    rng = np.random.default_rng(21)
    for _ in range(3):
        mesh, depth = C.random_body(rng, 150, 700)
        out.append(C.Case(mesh, np.array([0.7]), np.array([0.0]), C.six_dofs(), C.six_dofs(), depth=depth))
    return out


def _items(cases, seed=3, n=14):
    rng = np.random.default_rng(seed)
    body = rng.integers(0, len(cases), n)
    body[:len(cases)] = np.arange(len(cases))          # every body at least once
    rng.shuffle(body)
    omega = rng.uniform(0.3, 2.2, n)
    return body, omega


def _rhs(case, omega, beta=30.0):
    c = C.Case(case.mesh, np.array([omega]), np.array([beta]), case.rad, case.force, rho=case.rho, g=case.g,
               depth=case.depth)
    return C.body_conditions(c)   # (2^s N, 1 + ndof)


def _single(case, mode, omegas, nvels):
    with nb.Solver(0, mode) as s:
        s.set_case(case)
        nds = C.generalised_normals(case)
        return [s.solve_frequencies(np.array([w]), v[:, :, None], nds)[:, :, 0] for w, v in zip(omegas, nvels)]


@pytest.mark.parametrize("env", [{}, {"NEMOH_B200_BATCH_BYTES": str(48 << 20)},
                                 {"NEMOH_B200_RANKINE_CACHE_BYTES": "0"}],
                         ids=["one_batch", "split_batches", "per_slot_rankine"])
def test_bodies_match_single_body_path(env):
    """The single-body path reads the mesh's Rankine cache; the bodies read
    their own caches, or (cache budget 0) evaluate the Rankine part per slot."""
    B.build()
    cases = _bodies()
    body, omega = _items(cases)
    nvels = [_rhs(cases[b], w) for b, w in zip(body, omega)]
    old = {k: os.environ.get(k) for k in env}
    os.environ.update(env)
    try:
        got = {}
        for mode in (nb.FP64, nb.MIXED):
            with nb.Solver(0, mode) as s:
                ids = [s.add_body(c) for c in cases]
                assert ids == list(range(len(cases)))
                got[mode] = s.solve_bodies(body, omega, nvels)
    finally:
        for k, v in old.items():
            if v is None:
                del os.environ[k]
            else:
                os.environ[k] = v
    for b in range(len(cases)):
        sel = [i for i in range(len(body)) if body[i] == b]
        ref64 = _single(cases[b], nb.FP64, omega[sel], [nvels[i] for i in sel])
        refmx = _single(cases[b], nb.MIXED, omega[sel], [nvels[i] for i in sel])
        for q, i in enumerate(sel):
            scale = np.abs(ref64[q]).max()
            assert np.abs(got[nb.FP64][i] - ref64[q]).max() <= 1e-12 * scale, (cases[b].name, i)
            assert np.abs(got[nb.MIXED][i] - refmx[q]).max() <= 1e-10 * scale, (cases[b].name, i)
        F = np.stack([got[nb.MIXED][i] for i in sel], axis=2)
        F64 = np.stack(ref64, axis=2)
        assert G.coef_err(F, F64, 1) < 1e-6


def test_bodies_refuse_unknown_body_and_keep_working():
    B.build()
    cases = _bodies()[:2]
    with nb.Solver(0, nb.FP64) as s:
        for c in cases:
            s.add_body(c)
        nv = _rhs(cases[0], 0.9)
        with pytest.raises(nb.NemohError):
            s.solve_bodies(np.array([0, 5]), np.array([0.9, 0.9]), [nv, nv])
        out = s.solve_bodies(np.array([0]), np.array([0.9]), [nv])
        ref = _single(cases[0], nb.FP64, [0.9], [nv])[0]
        assert np.abs(out[0] - ref).max() <= 1e-12 * np.abs(ref).max()


def test_requests_with_device_rhs_match_host_rhs():
    """nemoh_b200_solve_requests builds each request's right-hand sides on the
    device (pre-processor formulas); its forces equal those of
    nemoh_b200_solve_bodies given the host pre-processor's right-hand sides
    for the same (body, omega, heading), within 1e-12 of the largest force."""
    B.build()
    cases = _bodies()
    body, omega = _items(cases, seed=8, n=12)
    beta = np.random.default_rng(9).uniform(0.0, 180.0, len(body))
    nvels = [_rhs(cases[b], w, be) for b, w, be in zip(body, omega, beta)]
    for mode in (nb.FP64, nb.MIXED):
        with nb.Solver(0, mode) as s:
            for c in cases:
                bid = s.add_body(c)
                s.set_body_dofs(bid, c.rad)
            got = s.solve_requests(body, omega, np.radians(beta))
            ref = s.solve_bodies(body, omega, nvels)
        # mixed precision: both sides refined to a 1e-12 residual, not bitwise
        tol = 1e-12 if mode == nb.FP64 else 1e-10
        for g, r in zip(got, ref):
            assert g.shape == r.shape
            assert np.abs(g - r).max() <= tol * np.abs(r).max()


@pytest.mark.parametrize("mode", [nb.FP64, nb.MIXED], ids=["fp64", "mixed"])
def test_graph_replay_matches_direct_launches(mode):
    """Graph mode: the first batch runs its launches directly, the second
    identical batch is captured into a CUDA graph and the later ones replay
    it; every call gives the direct path's forces (1e-12 of the largest force
    in FP64, 1e-10 in mixed precision, where the refinement's last bits
    differ)."""
    B.build()
    cases = _bodies()
    body, omega = _items(cases, seed=5, n=10)
    nvels = [_rhs(cases[b], w) for b, w in zip(body, omega)]
    with nb.Solver(0, mode) as s:
        for c in cases:
            s.add_body(c)
        ref = s.solve_bodies(body, omega, nvels)
        s.set_graphs(True)
        runs = [s.solve_bodies(body, omega, nvels) for _ in range(4)]
        cap, rep = s.graph_stats()
    assert cap >= 1 and rep >= 2, (cap, rep)
    tol = 1e-12 if mode == nb.FP64 else 1e-10
    for got in runs:
        for g, r in zip(got, ref):
            assert np.abs(g - r).max() <= tol * np.abs(r).max()


def test_fallback_in_a_ragged_batch():
    """With the refinement cut to one pass, systems of a cross-body batch miss
    the 1e-12 residual and are re-solved with FP64 factors (only those, when
    some converged); the results stay within 1e-6 per coefficient of FP64."""
    B.build()
    cases = _bodies()
    body, omega = _items(cases, seed=13, n=12)
    nvels = [_rhs(cases[b], w) for b, w in zip(body, omega)]
    old = os.environ.get("NEMOH_B200_REFINE_MAX_IT")
    os.environ["NEMOH_B200_REFINE_MAX_IT"] = "1"
    try:
        with nb.Solver(0, nb.MIXED) as s:
            for c in cases:
                s.add_body(c)
            got = s.solve_bodies(body, omega, nvels)
            batches, systems = s.fallback_count()
    finally:
        if old is None:
            del os.environ["NEMOH_B200_REFINE_MAX_IT"]
        else:
            os.environ["NEMOH_B200_REFINE_MAX_IT"] = old
    assert batches >= 1
    with nb.Solver(0, nb.FP64) as s:
        for c in cases:
            s.add_body(c)
        ref = s.solve_bodies(body, omega, nvels)
    for b in range(len(cases)):
        sel = [i for i in range(len(body)) if body[i] == b]
        F = np.stack([got[i] for i in sel], axis=2)
        F64 = np.stack([ref[i] for i in sel], axis=2)
        assert G.coef_err(F, F64, 1) < 1e-6, cases[b].name


def test_prepared_bodies_match_lazy_caches():
    """nemoh_b200_prepare_bodies evaluates every body's Rankine parts up front;
    the solves afterwards (with autotuning off, the default sweep) equal those
    of a context that evaluates them at first use, within 1e-12 of the largest
    force."""
    B.build()
    cases = _bodies()
    body, omega = _items(cases, seed=12, n=10)
    nvels = [_rhs(cases[b], w) for b, w in zip(body, omega)]
    out = {}
    for prepared in (False, True):
        with nb.Solver(0, nb.FP64) as s:
            for c in cases:
                s.add_body(c)
            if prepared:
                s.prepare_bodies()
                nb.set_autotune(False)
            try:
                out[prepared] = s.solve_bodies(body, omega, nvels)
            finally:
                nb.set_autotune(True)
    for a, b in zip(out[True], out[False]):
        assert np.abs(a - b).max() <= 1e-12 * np.abs(b).max()
