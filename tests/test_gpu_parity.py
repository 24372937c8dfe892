"""Parity of the CUDA path with the CPU FP64 oracle, through the C-ABI.

Tolerances (FP64 path): panel geometry bit-exact (it decides every branch);
Green tables 1e-13 of the table's magnitude; influence matrices 1e-12 of each
row's largest entry in deep water and 1e-10 in finite depth (the exponential
image sums cancel more; a flipped branch would show as ~1e-3); source
strengths and potentials 1e-10; forces (added mass, damping, excitation)
1e-9 per coefficient (gpu_cases.parity_err: each coefficient against itself,
floored at 1e-6 of its family's largest value; families that vanish by
symmetry within 1e-12 of their kind's largest coefficient) and 1e-11 of the
largest force of each integration case. Mixed precision (FP32 LU + FP64
refinement): 1e-6 of FP64.
"""
import os

import numpy as np
import pytest

import gpu_cases as G
import nemoh_b200 as nb
import oracle_lib as O
import verification as V
from nemoh_b200 import build as B
from nemoh_b200 import cases as C

pytestmark = pytest.mark.gpu

CASES = G.small_cases()
IDS = [c.name for c in CASES]


@pytest.fixture(scope="module")
def solver():
    B.build()
    s = nb.Solver(0, nb.FP64)
    yield s
    s.close()


def _mesh(s, case):
    m = case.mesh
    s.set_mesh(m.nodes, m.panels, m.isym, case.rho, case.g, case.depth)


@pytest.mark.parametrize("case", CASES, ids=IDS)
def test_geometry_bit_exact(solver, case):
    _mesh(solver, case)
    g, zer = solver.geometry()
    o = G.oracle_for(case)
    go, zo = o.geometry()
    assert zer == zo
    assert np.array_equal(g, go), np.abs(g - go).max()


def test_tables_match_oracle(solver):
    xr, xz, apd = solver.tables()
    case = CASES[0]
    o = G.oracle_for(case)
    xr2, xz2, apd2 = o.tables()
    assert np.array_equal(xr, xr2) and np.array_equal(xz, xz2)
    scale = np.abs(apd2).max(axis=(1, 2), keepdims=True)
    assert np.max(np.abs(apd - apd2) / scale) < 1e-13


@pytest.mark.parametrize("case", CASES, ids=IDS)
def test_assembly_matches_oracle(solver, case):
    _mesh(solver, case)
    o = G.oracle_for(case)
    for w in case.omegas:
        gm, mode = solver.assemble(w)
        om, mode_o, _ = o.assemble(w)
        assert mode == mode_o
        tol = 1e-10 if mode else 1e-12
        for a, b in zip(gm, om):
            row = np.abs(b).max(axis=1, keepdims=True)
            err = np.abs(a - b) / row
            assert err.max() < tol, (case.name, w, err.max(), np.unravel_index(err.argmax(), err.shape))


@pytest.mark.parametrize("case", CASES, ids=IDS)
def test_solve_problem_matches_oracle(solver, case):
    """The reference boundary, problem by problem in the pre-processor's order."""
    _mesh(solver, case)
    o = G.oracle_for(case)
    nv = C.body_conditions(case)
    npb = len(case.betas_deg) + len(case.rad)
    for j in range(nv.shape[1]):
        w = case.omegas[j // npb]
        T = 2 * np.pi / w
        g = solver.solve_potential(T, nv[:, j])
        r = o.solve_problem(T, nv[:, j])
        assert g["nexp"] == r["nexp"]
        for k in ("zigb", "zpb") + (("zigs", "zps") if case.mesh.isym else ()):
            scale = np.abs(r[k]).max()
            assert np.abs(g[k] - r[k]).max() <= 1e-10 * scale, (case.name, j, k)


@pytest.mark.parametrize("case", CASES, ids=IDS)
def test_forces_match_oracle(solver, case, tmp_path):
    _mesh(solver, case)
    nvel, nds, npb = G.problems(case)
    F = solver.solve_frequencies(case.omegas, nvel, nds)
    Fo = G.oracle_forces(case, str(tmp_path))
    assert G.parity_err(F, Fo, len(case.betas_deg)) < G.PARITY_TOL
    assert G.rel_err(F, Fo) < 1e-11


def test_two_body_finite_depth_verification_case(solver, tmp_path):
    fx = V.load("2Bodies")
    case = V.case_from_fixture(fx, omegas=fx["omegas"][4:7])
    _mesh(solver, case)
    nvel, nds, npb = G.problems(case)
    F = solver.solve_frequencies(case.omegas, nvel, nds)
    Fo = G.oracle_forces(case, str(tmp_path))
    assert G.parity_err(F, Fo, len(case.betas_deg)) < G.PARITY_TOL
    assert G.rel_err(F, Fo) < 1e-11


def test_cylinder_verification_against_reference_results(solver):
    fx = V.load("Cylinder")
    case = V.case_from_fixture(fx)
    _mesh(solver, case)
    nvel, nds, npb = G.problems(case)
    F = solver.solve_frequencies(case.omegas, nvel, nds)
    nb_ = len(case.betas_deg)
    A = np.zeros((len(case.omegas), F.shape[0], len(case.rad)))
    Bd = np.zeros_like(A)
    for iw, w in enumerate(case.omegas):
        A[iw] = F[:, nb_:, iw].imag / w
        Bd[iw] = -F[:, nb_:, iw].real
    errs = V.compare_cw(fx, A, Bd)
    assert max(errs)[0] < 1e-4


def _lu_launches(n, nb=32, outer=128):
    """Launches of the two-level FP64 LU: per 32-column step the diagonal
    block and the panel, plus the updates inside the 128-column panel and its
    row strip; one trailing update per panel."""
    count = 0
    for k0 in range(0, n, outer):
        kend = min(k0 + outer, n)
        for k in range(k0, kend, nb):
            count += 2
            if k + min(nb, n - k) < kend:
                count += 1 + (kend < n)
        count += kend < n
    return count


def test_repeated_frequency_reuses_factorization(solver):
    case = CASES[0]
    _mesh(solver, case)
    nv = C.body_conditions(case)
    T = 2 * np.pi / case.omegas[0]
    n0 = solver.launches
    solver.solve_potential(T, nv[:, 0])
    n1 = solver.launches
    solver.solve_potential(T, nv[:, 1])
    n2 = solver.launches
    # the second call launches no assembly and no factorization: two assembly
    # launches (Rankine and wave passes), the LU launches and one diagonal-block
    # inversion fewer
    assert (n1 - n0) - (n2 - n1) == 3 + _lu_launches(case.mesh.npanels)


def test_degenerate_panel_reports_status(solver):
    case = CASES[0]
    panels = case.mesh.panels.copy()
    panels[5] = [panels[5][0]] * 4
    with pytest.raises(nb.NemohError) as e:
        solver.set_mesh(case.mesh.nodes, panels, 0, 1025.0, 9.81, 0.0)
    assert e.value.code == 2


def test_tiny_frequency_reports_status(solver):
    case = CASES[0]
    _mesh(solver, case)
    nv = C.body_conditions(case)
    with pytest.raises(nb.NemohError) as e:
        solver.solve_potential(2 * np.pi / 5e-5, nv[:, 0])
    assert e.value.code == 4


def test_batched_sizes_refused(solver):
    """nrhs outside 1..16 and missing buffers are refused with the header's
    status codes, and the context solves as before afterwards. Every buffer
    passed is large enough for the call it is passed to."""
    import torch
    case = CASES[0]
    _mesh(solver, case)
    m = case.mesh
    nc = m.npanels * 2 ** m.isym
    rng = np.random.default_rng(11)
    nvel = rng.standard_normal((nc, 7, 1)) + 1j * rng.standard_normal((nc, 7, 1))
    nds = np.asfortranarray(rng.standard_normal((3, nc)))
    om = np.array([case.omegas[0]])
    before = solver.solve_frequencies(om, nvel, nds)
    lib = nb.load_library()
    d = lambda a: a.ctypes.data_as(nb._d)
    h = solver._h
    big = np.zeros((nc, 17, 1), np.complex128, order="F")
    force = np.zeros((3, 17, 1), np.complex128, order="F")
    assert lib.nemoh_b200_solve_frequencies(h, 1, d(om), 0, d(big), 3, d(nds), d(force)) == 1
    assert lib.nemoh_b200_solve_frequencies(h, 1, d(om), 17, d(big), 3, d(nds), d(force)) == 23
    assert "1..16" in lib.nemoh_b200_last_error(h).decode()
    assert lib.nemoh_b200_solve_frequencies(h, 1, d(om), 7, d(big), 3, None, d(force)) == 1
    dev = torch.zeros(2 * nc * 17, dtype=torch.float64, device="cuda:0")
    dnds = torch.zeros(3 * nc, dtype=torch.float64, device="cuda:0")
    dforce = torch.zeros(2 * 3 * 17, dtype=torch.float64, device="cuda:0")
    assert lib.nemoh_b200_solve_frequencies_device(h, 1, d(om), 0, dev.data_ptr(), 3, dnds.data_ptr(),
                                                   dforce.data_ptr(), None) == 1
    # host buffers handed in as device memory: refused before any launch
    launches = solver.launches
    assert lib.nemoh_b200_solve_frequencies_device(h, 1, d(om), 7, nvel.ctypes.data, 3, dnds.data_ptr(),
                                                   dforce.data_ptr(), None) == 1
    assert "nvel_device: host memory" in lib.nemoh_b200_last_error(h).decode()
    assert lib.nemoh_b200_solve_frequencies_device(h, 1, d(om), 7, dev.data_ptr(), 3, dnds.data_ptr(),
                                                   force.ctypes.data, None) == 1
    assert "force_device" in lib.nemoh_b200_last_error(h).decode()
    assert solver.launches == launches
    torch.cuda.synchronize()
    after = solver.solve_frequencies(om, nvel, nds)
    np.testing.assert_allclose(after, before, rtol=0, atol=1e-12 * np.abs(before).max())


def _first_panels(case, k):
    """The case restricted to its first k panels (an open surface): orders
    below, at and just above the tile and panel widths of the kernels."""
    m = case.mesh
    sub = C.Mesh(m.nodes, m.panels[:k], m.isym)
    c = C.Case(sub, case.omegas[:2], case.betas_deg[:1], case.rad, case.force, rho=case.rho, g=case.g,
               depth=case.depth)
    c.name = "%s_first%d" % (case.name, k)
    return c


TINY = [(0, 1), (0, 17), (0, 129), (0, 257), (1, 5), (1, 33), (1, 65)]


@pytest.mark.parametrize("which,k", TINY, ids=["%s_%d" % (IDS[w], k) for w, k in TINY])
def test_small_and_ragged_orders_match_oracle(which, k, tmp_path):
    """FP64 forces against the oracle (1e-9 of the largest force) and mixed
    precision against FP64 (1e-6) for a single panel and for orders one above
    a multiple of the 16-row assembly tiles, the 32-column LU steps, the
    64-row triangular-solve blocks and the 128-column outer panels (129 and
    257: tensor-core outer updates of one row and column)."""
    case = _first_panels(CASES[which], k)
    with nb.Solver(0, nb.FP64) as s64, nb.Solver(0, nb.MIXED) as smx:
        for s in (s64, smx):
            _mesh(s, case)
        nvel, nds, npb = G.problems(case)
        F64 = s64.solve_frequencies(case.omegas, nvel, nds)
        Fmx = smx.solve_frequencies(case.omegas, nvel, nds)
    Fo = G.oracle_forces(case, str(tmp_path))
    scale = np.abs(Fo).max()
    assert scale > 0
    assert np.abs(F64 - Fo).max() <= 1e-9 * scale, (case.name, np.abs(F64 - Fo).max() / scale)
    assert np.abs(Fmx - F64).max() <= 1e-6 * scale, (case.name, np.abs(Fmx - F64).max() / scale)


@pytest.mark.parametrize("which", [0, 1], ids=[IDS[0], IDS[1]])
def test_sixteen_problems_per_frequency(which, tmp_path):
    """The largest batch of right-hand sides (10 headings + 6 DOF = 16 per
    frequency): FP64 against the oracle, mixed against FP64."""
    base = CASES[which]
    case = C.Case(base.mesh, base.omegas[:2], np.linspace(0.0, 162.0, 10), base.rad, base.force, rho=base.rho,
                  g=base.g, depth=base.depth)
    case.name = base.name + "_16rhs"
    with nb.Solver(0, nb.FP64) as s64, nb.Solver(0, nb.MIXED) as smx:
        for s in (s64, smx):
            _mesh(s, case)
        nvel, nds, npb = G.problems(case)
        assert npb == 16
        F64 = s64.solve_frequencies(case.omegas, nvel, nds)
        Fmx = smx.solve_frequencies(case.omegas, nvel, nds)
    Fo = G.oracle_forces(case, str(tmp_path))
    assert G.parity_err(F64, Fo, len(case.betas_deg)) < G.PARITY_TOL
    assert G.rel_err(Fmx, F64) < 1e-6


def test_two_spheres_8000_panels_mixed_matches_fp64():
    """The precision configuration at full size: two floating spheres of radius
    4 m, 20 m apart, 8,000 panels, deep water, 12 DOF + 2 headings, at the
    lowest, a middle and the highest of its 30 frequencies: mixed precision
    (split-BF16 tensor-core LU + FP64 refinement) within 1e-6 of FP64 per
    integration case. The oracle is too slow at this order; its parity with
    the FP64 path is covered at the smaller orders above."""
    import dataclasses
    case = C.config_two_spheres()
    case = dataclasses.replace(case, omegas=case.omegas[[0, 15, 29]])
    assert case.mesh.npanels == 8000
    with nb.Solver(0, nb.FP64) as s64, nb.Solver(0, nb.MIXED) as smx:
        for s in (s64, smx):
            _mesh(s, case)
        nvel, nds, npb = G.problems(case)
        assert npb == 14
        F64 = s64.solve_frequencies(case.omegas, nvel, nds)
        Fmx = smx.solve_frequencies(case.omegas, nvel, nds)
        it, res = smx.last_refinement()
    assert np.isfinite(F64).all() and np.abs(F64).max() > 0
    assert G.rel_err(Fmx, F64) < 1e-6, (G.rel_err(Fmx, F64), it, res)


@pytest.mark.parametrize("case", CASES, ids=IDS)
def test_mixed_precision_matches_fp64(case):
    with nb.Solver(0, nb.FP64) as s64, nb.Solver(0, nb.MIXED) as smx:
        for s in (s64, smx):
            _mesh(s, case)
        nvel, nds, npb = G.problems(case)
        F64 = s64.solve_frequencies(case.omegas, nvel, nds)
        Fmx = smx.solve_frequencies(case.omegas, nvel, nds)
        assert G.rel_err(Fmx, F64) < 1e-6
        # a good low-precision factorization converges in a few refinement steps
        it, res = smx.last_refinement()
        assert it <= 6 and res <= 1e-12, (it, res)


def test_mixed_fallback_to_fp64_factors(tmp_path):
    """Refinement capped at one iteration cannot reach 1e-12: the batch is
    re-solved with FP64 factors on the device and matches the FP64 path."""
    import subprocess
    import sys
    case = CASES[1]
    script = tmp_path / "fallback.py"
    script.write_text(
        "import sys, numpy as np\n"
        "sys.path[:0] = %r\n"
        "import gpu_cases as G, nemoh_b200 as nb\n"
        "case = [c for c in G.small_cases() if c.name == %r][0]\n"
        "nvel, nds, npb = G.problems(case)\n"
        "m = case.mesh\n"
        "out = {}\n"
        "for mode in (nb.FP64, nb.MIXED):\n"
        "    with nb.Solver(0, mode) as s:\n"
        "        s.set_mesh(m.nodes, m.panels, m.isym, case.rho, case.g, case.depth)\n"
        "        out[mode] = s.solve_frequencies(case.omegas, nvel, nds)\n"
        "        it = s.last_refinement()[0]\n"
        "print('ERR', G.rel_err(out[nb.MIXED], out[nb.FP64]), 'IT', it)\n"
        % ([str(p) for p in (B.HERE + "/..", B.HERE + "/../tests")], case.name))
    env = dict(os.environ, NEMOH_B200_REFINE_MAX_IT="1")
    r = subprocess.run([sys.executable, str(script)], env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    line = [l for l in r.stdout.splitlines() if l.startswith("ERR")][-1].split()
    assert float(line[1]) < 1e-10 and int(line[3]) == -1, line


def test_one_tile_per_cta_tensor_core_update(tmp_path):
    """The one-tile-per-CTA form of the tensor-core trailing update (the other
    tests run the default persistent form; NEMOH_B200_TC_PERSISTENT=0 is read
    once per process, hence a child process): the mixed path through it
    matches FP64 within 1e-6 per coefficient on orders with one and with
    several outer updates (the cylinder of 300 panels, a hemisphere of 640),
    with the refinement converging."""
    import subprocess
    import sys
    script = tmp_path / "persistent.py"
    script.write_text(
        "import sys, numpy as np\n"
        "sys.path[:0] = %r\n"
        "import gpu_cases as G, nemoh_b200 as nb\n"
        "from nemoh_b200 import cases as C\n"
        "cyl = C.config_cylinder(n_omega=3)\n"
        "sph = C.Case(C.hemisphere_mesh(3.0, 16, 40, jitter=0.2, rng=np.random.default_rng(7)),\n"
        "             np.array([0.5, 1.1, 1.7]), np.array([0.0]), C.six_dofs(), C.six_dofs(), depth=0.0)\n"
        "for case in (cyl, sph):\n"
        "    nvel, nds, npb = G.problems(case)\n"
        "    out = {}\n"
        "    for mode in (nb.FP64, nb.MIXED):\n"
        "        with nb.Solver(0, mode) as s:\n"
        "            s.set_case(case)\n"
        "            out[mode] = s.solve_frequencies(case.omegas, nvel, nds)\n"
        "            it = s.last_refinement()[0]\n"
        "    print('ERR', case.mesh.npanels, G.coef_err(out[nb.MIXED], out[nb.FP64], 1), 'IT', it)\n"
        % [str(p) for p in (B.HERE + "/..", B.HERE + "/../tests")])
    env = dict(os.environ, NEMOH_B200_TC_PERSISTENT="0")
    r = subprocess.run([sys.executable, str(script)], env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l.split() for l in r.stdout.splitlines() if l.startswith("ERR")]
    assert len(lines) == 2, r.stdout
    for line in lines:
        assert float(line[2]) < 1e-6 and 0 < int(line[4]) <= 6, line


def test_merged_outer_updates_match_separate_ones(tmp_path):
    """Mixed-precision LU with the outer updates of panel pairs merged (the
    default) and with one update per panel (NEMOH_B200_TC_MERGE=0, a child
    process: the switch is read once per process), on orders with 3 and 5
    outer panels and a ragged batch of both: the refinement converges in the
    same few passes without any FP64 fallback (a wrong factor would still give
    right answers through the fallback, so its count is checked), and the
    forces agree within 1e-10 of the largest force."""
    import subprocess
    import sys
    script = tmp_path / "merge.py"
    script.write_text(
        "import sys, numpy as np\n"
        "sys.path[:0] = %r\n"
        "import gpu_cases as G, nemoh_b200 as nb\n"
        "from nemoh_b200 import cases as C\n"
        "cyl = C.config_cylinder(n_omega=3)\n"
        "sph = C.Case(C.hemisphere_mesh(3.0, 16, 40, jitter=0.2, rng=np.random.default_rng(7)),\n"
        "             np.array([0.5, 1.1, 1.7]), np.array([0.0]), C.six_dofs(), C.six_dofs(), depth=0.0)\n"
        "res = {}\n"
        "for case in (cyl, sph):\n"
        "    nvel, nds, npb = G.problems(case)\n"
        "    with nb.Solver(0, nb.MIXED) as s:\n"
        "        s.set_case(case)\n"
        "        res[case.name] = s.solve_frequencies(case.omegas, nvel, nds)\n"
        "        res['it_' + case.name] = np.array(s.last_refinement()[0])\n"
        "        res['fb_' + case.name] = np.array(s.fallback_count())\n"
        "body = np.array([0, 1, 1, 0]); om = np.array([0.6, 0.9, 1.3, 1.9])\n"
        "nv = [C.body_conditions(C.Case((cyl, sph)[b].mesh, np.array([w]), np.array([20.0]), (cyl, sph)[b].rad,\n"
        "                               (cyl, sph)[b].force, depth=(cyl, sph)[b].depth)) for b, w in zip(body, om)]\n"
        "with nb.Solver(0, nb.MIXED) as s:\n"
        "    for c in (cyl, sph):\n"
        "        s.add_body(c)\n"
        "    for i, f in enumerate(s.solve_bodies(body, om, nv)):\n"
        "        res['bodies_%%d' %% i] = f\n"
        "    res['fb_bodies'] = np.array(s.fallback_count())\n"
        "np.savez(sys.argv[1], **res)\n"
        % [str(p) for p in (B.HERE + "/..", B.HERE + "/../tests")])
    got = {}
    for form, env in (("merged", {}), ("separate", {"NEMOH_B200_TC_MERGE": "0"})):
        out = tmp_path / (form + ".npz")
        r = subprocess.run([sys.executable, str(script), str(out)], env=dict(os.environ, **env),
                           capture_output=True, text=True, timeout=600)
        assert r.returncode == 0, r.stderr[-2000:]
        got[form] = dict(np.load(out))
    a, b = got["merged"], got["separate"]
    for k in a:
        if k.startswith("fb_"):
            assert tuple(a[k]) == (0, 0) and tuple(b[k]) == (0, 0), (k, a[k], b[k])
        elif k.startswith("it_"):
            assert 0 < int(a[k]) <= 4 and abs(int(a[k]) - int(b[k])) <= 1, (k, a[k], b[k])
        else:
            scale = np.abs(b[k]).max()
            assert np.abs(a[k] - b[k]).max() <= 1e-10 * scale, (k, np.abs(a[k] - b[k]).max() / scale)


def test_dataflow_and_cluster_sweeps_agree(tmp_path):
    """The two triangular sweeps, each forced in a child process
    (NEMOH_B200_SWEEP is read once per process): FP64 forces agree within
    1e-12 of the largest force, the mixed ones match FP64 within 1e-6 per
    coefficient with the refinement converging, on a cylinder of 300 panels
    (5 row blocks, 2 with symmetry classes) and a hemisphere of 640 (10 row
    blocks, one partial), and a cross-body batch of both (a ragged sweep)."""
    import subprocess
    import sys
    script = tmp_path / "sweeps.py"
    script.write_text(
        "import sys, numpy as np\n"
        "sys.path[:0] = %r\n"
        "import gpu_cases as G, nemoh_b200 as nb\n"
        "from nemoh_b200 import cases as C\n"
        "cyl = C.config_cylinder(n_omega=3)\n"
        "sph = C.Case(C.hemisphere_mesh(3.0, 16, 40, jitter=0.2, rng=np.random.default_rng(7)),\n"
        "             np.array([0.5, 1.1, 1.7]), np.array([0.0]), C.six_dofs(), C.six_dofs(), depth=0.0)\n"
        "res = {}\n"
        "for case in (cyl, sph):\n"
        "    nvel, nds, npb = G.problems(case)\n"
        "    for mode in (nb.FP64, nb.MIXED):\n"
        "        with nb.Solver(0, mode) as s:\n"
        "            s.set_case(case)\n"
        "            res['%%s_%%d' %% (case.name, mode)] = s.solve_frequencies(case.omegas, nvel, nds)\n"
        "            res['it_%%s_%%d' %% (case.name, mode)] = np.array(s.last_refinement()[0])\n"
        "body = np.array([0, 1, 0, 1]); om = np.array([0.6, 0.9, 1.3, 1.9])\n"
        "nv = []\n"
        "for b, w in zip(body, om):\n"
        "    c = (cyl, sph)[b]\n"
        "    nv.append(C.body_conditions(C.Case(c.mesh, np.array([w]), np.array([20.0]), c.rad, c.force,\n"
        "                                       rho=c.rho, g=c.g, depth=c.depth)))\n"
        "for mode in (nb.FP64, nb.MIXED):\n"
        "    with nb.Solver(0, mode) as s:\n"
        "        for c in (cyl, sph):\n"
        "            s.add_body(c)\n"
        "        out = s.solve_bodies(body, om, nv)\n"
        "        for i, f in enumerate(out):\n"
        "            res['bodies_%%d_%%d' %% (i, mode)] = f\n"
        "np.savez(sys.argv[1], **res)\n"
        % [str(p) for p in (B.HERE + "/..", B.HERE + "/../tests")])
    got = {}
    for form in ("flow", "cluster"):
        env = dict(os.environ, NEMOH_B200_SWEEP=form)
        out = tmp_path / (form + ".npz")
        r = subprocess.run([sys.executable, str(script), str(out)], env=env, capture_output=True, text=True,
                           timeout=600)
        assert r.returncode == 0, r.stderr[-2000:]
        got[form] = dict(np.load(out))
    a, b = got["flow"], got["cluster"]
    assert set(a) == set(b)
    for k in a:
        if k.startswith("it_"):
            assert 0 < int(a[k]) <= 6 or k.endswith("_%d" % nb.FP64), (k, a[k])
            continue
        scale = np.abs(b[k]).max()
        tol = 1e-12 if k.endswith("_%d" % nb.FP64) else 1e-6
        assert np.abs(a[k] - b[k]).max() <= tol * scale, (k, np.abs(a[k] - b[k]).max() / scale)
    for k in a:
        if k.endswith("_%d" % nb.MIXED) and not k.startswith("it_"):
            ref = a[k[:-len(str(nb.MIXED))] + str(nb.FP64)]
            if ref.ndim == 3:
                assert G.coef_err(a[k], ref, 1) < 1e-6, k
                assert G.coef_err(b[k], ref, 1) < 1e-6, k


def test_dataflow_sweep_wait_runs_out_and_device_stays_usable(solver):
    """A dataflow sweep whose only item waits on a ready flag that nothing
    raises: the bounded wait ends with the sweep-timeout status (31) in well
    under the test's time, and a solve on the same device afterwards still
    matches the oracle."""
    st, ms = nb.sweep_timeout_check(0)
    assert st == 31, st
    assert ms < 30000.0, ms
    case = CASES[0]
    _mesh(solver, case)
    o = G.oracle_for(case)
    nv = C.body_conditions(case)
    T = 2 * np.pi / case.omegas[0]
    g = solver.solve_potential(T, nv[:, 0])
    r = o.solve_problem(T, nv[:, 0])
    assert np.abs(g["zpb"] - r["zpb"]).max() <= 1e-10 * np.abs(r["zpb"]).max()


@pytest.mark.parametrize("case", CASES, ids=IDS)
def test_kochin_matches_oracle(solver, case):
    """COMPUTE_KOCHIN on the GPU vs the oracle, on the same source strengths:
    every direction within 1e-9 of the problem's largest |H| (the force
    tolerance; the panel sum cancels, so last-place differences of exp and of
    the complex divisions grow to ~1e-11)."""
    _mesh(solver, case)
    o = G.oracle_for(case)
    nv = C.body_conditions(case)
    npb = len(case.betas_deg) + len(case.rad)
    theta = np.linspace(0.0, 2.0 * np.pi, 37)
    for w_idx in (0, len(case.omegas) - 1):
        T = 2 * np.pi / case.omegas[w_idx]
        cols = range(w_idx * npb, (w_idx + 1) * npb)
        res = [solver.solve_potential(T, nv[:, j]) for j in cols]
        zigb = np.stack([r["zigb"] for r in res], axis=1)
        zigs = np.stack([r["zigs"] for r in res], axis=1)
        H = solver.kochin(T, theta, zigb, zigs, xeff=1.5, yeff=-0.5)
        Ho = o.kochin(T, theta, zigb, zigs if case.mesh.isym else None, xeff=1.5, yeff=-0.5)
        scale = np.abs(Ho).max(axis=0)
        assert np.all(scale > 0)
        err = (np.abs(H - Ho) / scale).max()
        assert err < 1e-9, (case.name, w_idx, err)


@pytest.mark.parametrize("which", ["cylinder300_deep", "barge_half_fd50", "two_bodies_fd"])
def test_device_body_conditions_match_preprocessor(solver, which):
    """NVEL, NDS and Froude-Krylov forces computed on the GPU against the
    pre-processor restatement in nemoh_b200.cases (1e-12 of each array's max)."""
    import dataclasses
    if which == "two_bodies_fd":
        fx = V.load("2Bodies")
        case = V.case_from_fixture(fx, omegas=fx["omegas"][4:7])
        case = dataclasses.replace(case, betas_deg=np.array([0.0, 30.0]), xeff=2.0, yeff=-1.0)
    else:
        case = [c for c in CASES if c.name == which][0]
        case = dataclasses.replace(case, betas_deg=np.array([0.0, 45.0, 120.0]), xeff=5.0, yeff=3.0)
    _mesh(solver, case)
    nvel, nds, fk = solver.body_conditions(case)
    nv0, nds0, fk0 = C.body_conditions(case), C.generalised_normals(case), C.froude_krylov(case)
    for got, ref in ((nvel, nv0), (nds, nds0), (fk, fk0)):
        assert got.shape == ref.shape
        assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max(), which


@pytest.mark.parametrize("which", [0, 1], ids=[IDS[0], IDS[1]])
def test_device_pointer_entry_points_match_host(solver, which):
    """Body conditions and the batched solve with device-resident buffers on a
    caller's stream give the host-buffer results: NVEL and NDS identical,
    Froude-Krylov forces (atomic sums) and forces (atomic mat-vec sums) within
    1e-12 of their largest entry."""
    import dataclasses
    import torch
    case = dataclasses.replace(CASES[which], betas_deg=np.array([0.0, 60.0]))
    _mesh(solver, case)
    nvel_h, nds_h, fk_h = solver.body_conditions(case)
    nc = case.mesh.npanels * 2 ** case.mesh.isym
    nw, nb, nr, nf = len(case.omegas), len(case.betas_deg), len(case.rad), len(case.force)
    dev = torch.device("cuda:0")
    stream = torch.cuda.Stream(dev)
    nvel_d = torch.zeros(2 * nc * (nb + nr) * nw, dtype=torch.float64, device=dev)
    nds_d = torch.zeros(nf * nc, dtype=torch.float64, device=dev)
    fk_d = torch.zeros(2 * nf * nb * nw, dtype=torch.float64, device=dev)
    force_d = torch.zeros(2 * nf * (nb + nr) * nw, dtype=torch.float64, device=dev)
    stream.wait_stream(torch.cuda.current_stream(dev))
    solver.body_conditions_device(case, nvel_d.data_ptr(), nds_d.data_ptr(), fk_d.data_ptr(), stream.cuda_stream)
    solver.solve_frequencies_device(case.omegas, nvel_d.data_ptr(), nb + nr, nf, nds_d.data_ptr(),
                                    force_d.data_ptr(), stream.cuda_stream)
    stream.synchronize()
    nv = nvel_d.cpu().numpy().view(np.complex128).reshape((nc, nb + nr, nw), order="F")
    nd = nds_d.cpu().numpy().reshape((nf, nc), order="F")
    fk = fk_d.cpu().numpy().view(np.complex128).reshape((nf, nb, nw), order="F")
    assert np.array_equal(nv.reshape(nc, -1, order="F"), nvel_h)
    assert np.array_equal(nd, nds_h)
    assert np.abs(fk.transpose(2, 1, 0) - fk_h).max() <= 1e-12 * np.abs(fk_h).max()
    F_h = solver.solve_frequencies(case.omegas, nv, nd)
    F_d = force_d.cpu().numpy().view(np.complex128).reshape((nf, nb + nr, nw), order="F")
    assert np.abs(F_d - F_h).max() <= 1e-12 * np.abs(F_h).max()


def _fs_points(case):
    """Points (x, y) on z = 0 around the body: a polar grid from just outside
    the waterline (tabulated wave term) to 30 body radii (asymptotic form)."""
    nodes = case.mesh.nodes
    r0 = np.hypot(nodes[:, 0], nodes[:, 1]).max()
    rr = r0 * np.array([1.15, 1.6, 3.0, 8.0, 30.0])
    th = np.linspace(0.0, 2.0 * np.pi, 13)[:-1] + 0.1
    R, TH = np.meshgrid(rr, th)
    return np.stack([(R * np.cos(TH)).ravel(), (R * np.sin(TH)).ravel()], axis=1)


@pytest.mark.parametrize("case", CASES, ids=IDS)
def test_free_surface_matches_oracle(solver, case):
    """Free-surface elevation (COMPUTE_POTENTIAL_DOMAIN on z = 0, ETA = i W/G PHI)
    on the GPU vs the oracle for the same source strengths: every point within
    1e-9 of the problem's largest |ETA| (the panel sums cancel like Kochin's)."""
    _mesh(solver, case)
    o = G.oracle_for(case)
    nv = C.body_conditions(case)
    npb = len(case.betas_deg) + len(case.rad)
    xy = _fs_points(case)
    for w_idx in (0, len(case.omegas) - 1):
        T = 2 * np.pi / case.omegas[w_idx]
        cols = range(w_idx * npb, (w_idx + 1) * npb)
        res = [solver.solve_potential(T, nv[:, j]) for j in cols]
        zigb = np.stack([r["zigb"] for r in res], axis=1)
        zigs = np.stack([r["zigs"] for r in res], axis=1)
        eta = solver.free_surface(T, xy, zigb, zigs)
        eo = o.free_surface(T, xy, zigb, zigs if case.mesh.isym else None)
        scale = np.abs(eo).max(axis=0)
        assert np.all(scale > 0)
        err = (np.abs(eta - eo) / scale).max()
        assert err < 1e-9, (case.name, w_idx, err)


def test_free_surface_more_problems_than_one_launch(solver):
    """More than 16 problems at once are taken 16 at a time: same values as
    one problem per call."""
    case = CASES[0]
    _mesh(solver, case)
    nv = C.body_conditions(case)
    T = 2 * np.pi / case.omegas[1]
    z = solver.solve_potential(T, nv[:, 0])["zigb"]
    rng = np.random.default_rng(3)
    zigb = z[:, None] * (rng.standard_normal(19) + 1j * rng.standard_normal(19))[None, :]
    xy = _fs_points(case)[:20]
    eta = solver.free_surface(T, xy, zigb)
    one = np.concatenate([solver.free_surface(T, xy, zigb[:, p]) for p in range(19)], axis=1)
    assert np.abs(eta - one).max() <= 1e-13 * np.abs(one).max()


def test_free_surface_and_kochin_match_stored_reference_values(solver):
    """The GPU path on the reference's Verification/Postprocessing case against
    its stored single-precision elevation (-i ETA) and Kochin function (i H):
    the tolerances of the oracle's own pin (2e-5 and 1e-4 of the largest stored
    modulus; 0.01 degree)."""
    fx = V.load("Postprocessing")
    case = V.case_from_fixture(fx)
    _mesh(solver, case)
    nv = C.body_conditions(case)
    T = 2 * np.pi / case.omegas[0]
    r = solver.solve_potential(T, nv[:, 0])
    fs = fx["freesurface"]
    pts, _ = C.freesurface_grid(*fx["fs_grid"])
    stored = np.array(fs["re"]) + 1j * np.array(fs["im"])
    eta = solver.free_surface(T, pts[fs["index"]], r["zigb"], r["zigs"])[:, 0]
    assert np.abs(-1j * eta - stored).max() < 2e-5 * np.abs(stored).max()
    k = fx["kochin"]
    Z = 1j * solver.kochin(T, np.radians(k["theta_deg"]), r["zigb"], r["zigs"])[:, 0]
    assert np.abs(np.abs(Z) - np.array(k["abs"])).max() < 1e-4 * np.max(k["abs"])
    dphi = (np.degrees(np.angle(Z)) - np.array(k["arg_deg"]) + 180.0) % 360.0 - 180.0
    assert np.abs(dphi).max() < 1e-2
