"""GPU: the serving layer (results alone == in the mix) and the drop-in driver."""
import os
import subprocess

import numpy as np
import pytest

import gpu_cases as G
import nemoh_b200 as nb
from nemoh_b200 import build as B
from nemoh_b200 import cases as C
from nemoh_b200 import serving as S

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.parametrize("precision", [nb.FP64, nb.MIXED])
def test_serving_result_same_alone_and_in_the_mix(precision):
    B.build()
    bodies = S.make_bodies(4, seed=11, n_min=150, n_max=400)
    srv = S.SolveServer(bodies, precision=precision, workers=2)
    try:
        reqs = S.make_requests(48, rate=0, n_bodies=4, seed=12)
        done, wall = srv.run(reqs, realtime=False)
        assert sorted(r.rid for r in done) == list(range(48))
        assert max(b[2] for b in srv.batches) > 1     # requests were batched
        assert max(b[1] for b in srv.batches) > 1     # with requests of different bodies together
        by = {r.rid: r for r in done}
        for rid in (0, 17, 33):
            r0 = reqs[rid]
            alone, _ = srv.run([S.Request(1000 + rid, r0.body, r0.omega, r0.beta_deg)], realtime=False)
            a, m = alone[0].force, by[rid].force
            tol = 1e-9 if precision == nb.FP64 else 1e-6
            assert np.abs(a - m).max() <= tol * np.abs(a).max()
    finally:
        srv.close()


def test_dropin_driver_matches_oracle(tmp_path):
    B.build()
    case = G.small_cases()[1]   # symmetric barge, finite depth
    ref = G.oracle_forces(case, str(tmp_path / "ref"))
    C.write_case(case, str(tmp_path / "gpu"))
    exe = os.path.join(ROOT, "nemoh_b200", "_build", "nemoh_solver_b200")
    subprocess.run([exe, str(tmp_path / "gpu")], check=True)
    F = np.loadtxt(str(tmp_path / "gpu" / "case" / "results" / "Forces.dat"), ndmin=2)
    got = G.decode_forces(case, F)
    assert G.parity_err(got, ref, len(case.betas_deg)) < G.PARITY_TOL


def _kochin_files(d, nprob):
    out = []
    for p in range(nprob):
        a = np.loadtxt(os.path.join(d, "case", "results", "Kochin.%5d.dat" % (p + 1)), ndmin=2)
        out.append(a[:, 1] * np.exp(1j * a[:, 2]))
    return a[:, 0], np.stack(out, axis=1)


def test_dropin_driver_kochin_files_match_oracle(tmp_path):
    """Kochin.<I5>.dat of every problem (symmetric finite-depth barge, wave
    measurement point off the origin) against the oracle's reference run."""
    import dataclasses
    import oracle_lib as O
    B.build()
    case = dataclasses.replace(G.small_cases()[1], kochin_theta=tuple(np.linspace(0.0, np.pi, 13)), xeff=3.0,
                               yeff=1.0)
    C.write_case(case, str(tmp_path / "ref"))
    O.run_case(str(tmp_path / "ref"))
    C.write_case(case, str(tmp_path / "gpu"))
    exe = os.path.join(ROOT, "nemoh_b200", "_build", "nemoh_solver_b200")
    subprocess.run([exe, str(tmp_path / "gpu")], check=True)
    th_r, Hr = _kochin_files(str(tmp_path / "ref"), case.nproblems)
    th_g, Hg = _kochin_files(str(tmp_path / "gpu"), case.nproblems)
    assert np.array_equal(th_r, th_g)
    err = (np.abs(Hg - Hr) / np.abs(Hr).max(axis=0)).max()
    assert err < 1e-9, err


def _fs_files(d, nprob):
    out = []
    for p in range(nprob):
        with open(os.path.join(d, "case", "results", "freesurface.%5d.dat" % (p + 1))) as f:
            head = [f.readline(), f.readline()]
        a = np.loadtxt(os.path.join(d, "case", "results", "freesurface.%5d.dat" % (p + 1)), skiprows=2,
                       max_rows=int(head[1].split("=")[1].split()[0]), ndmin=2)
        out.append(a[:, 4] + 1j * a[:, 5])
    return head, a[:, :2], np.stack(out, axis=1)


def test_dropin_driver_freesurface_files_match_oracle(tmp_path):
    """freesurface.<I5>.dat of every problem (deep-water cylinder, the
    pre-processor's 9 x 7 grid over 60 m x 40 m) against the oracle's reference
    run: same header, points and quadrangles, ETA within 1e-9 of the problem's
    largest |ETA|."""
    import dataclasses
    import oracle_lib as O
    B.build()
    case = dataclasses.replace(G.small_cases()[0], fs_grid=(9, 7, 60.0, 40.0))
    C.write_case(case, str(tmp_path / "ref"))
    O.run_case(str(tmp_path / "ref"))
    C.write_case(case, str(tmp_path / "gpu"))
    exe = os.path.join(ROOT, "nemoh_b200", "_build", "nemoh_solver_b200")
    subprocess.run([exe, str(tmp_path / "gpu")], check=True)
    hr, xr, Er = _fs_files(str(tmp_path / "ref"), case.nproblems)
    hg, xg, Eg = _fs_files(str(tmp_path / "gpu"), case.nproblems)
    assert hr == hg and np.array_equal(xr, xg) and xr.shape == (63, 2)
    qr = open(os.path.join(str(tmp_path / "ref"), "case", "results", "freesurface.%5d.dat" % 1)).read().split("\n")
    qg = open(os.path.join(str(tmp_path / "gpu"), "case", "results", "freesurface.%5d.dat" % 1)).read().split("\n")
    assert qr[2 + 63:] == qg[2 + 63:] and len(qr) == 2 + 63 + 48 + 1   # the quadrangles
    err = (np.abs(Eg - Er) / np.abs(Er).max(axis=0)).max()
    assert err < 1e-9, err
