"""The oracle's post-processor (postProcessor/Main.f90, Common/Results.f90,
postProcessor/IRF.f90).

Compute_IRF is checked against a known answer: a radiation kernel
K(t) = exp(-a t) has damping B(w) = a / (a^2 + w^2) and added mass
A(w) = A_inf - 1 / (a^2 + w^2) (Ogilvie's relations in the normalisation
K(t) = 2/pi int B(w) cos(w t) dw). From B and A sampled on 0.01..20 rad/s the
trapezoid sums must return K to the truncation of the frequency range and
A_inf to the truncation of the time range. The file outputs are checked
against the Forces.dat / FKForce.tec they were read from."""
import dataclasses
import math
import os

import numpy as np

import gpu_cases as G
import oracle_lib as O
from nemoh_b200 import cases as C


def test_irf_known_answer():
    a, a_inf = 0.8, 3.0
    w = np.linspace(0.01, 20.0, 2000)
    B = (a / (a * a + w * w))[:, None, None] * np.ones((1, 2, 3))
    A = (a_inf - 1.0 / (a * a + w * w))[:, None, None] * np.ones((1, 2, 3))
    K, ainf = O.irf(w, B, A, 400, 0.05)
    t = np.arange(400) * 0.05
    # the sampled range misses 2/pi int over [0, 0.01] and [20, inf) of B cos(wt):
    # at most 0.02 / (pi a) + 2 a / (20 pi) (reached at t = 0); the trapezoid rule adds
    # 3e-5 against the exact integral over the sampled range
    trunc = 0.02 / (math.pi * a) + 2 * a / (20 * math.pi)
    assert np.abs(K[:, 0, 0] - np.exp(-a * t)).max() < trunc + 1e-3
    assert np.abs(K - K[:, :1, :1]).max() == 0.0
    # the integral over [0.01, 20] itself, by scipy's oscillatory quadrature
    from scipy.integrate import quad
    for ti in (0.0, 1.0, 5.0, 19.95):
        ref = 2 / math.pi * quad(lambda x: a / (a * a + x * x), 0.01, 20.0, weight="cos", wvar=ti)[0]
        assert abs(K[int(round(ti / 0.05)), 0, 0] - ref) < 1e-4, ti
    assert np.allclose(ainf, ainf[0, 0]) and abs(ainf[0, 0] - a_inf) < 2e-2


def test_postprocessor_files(tmp_path):
    case = dataclasses.replace(G.small_cases()[0], irf=(0.1, 2.0), betas_deg=np.array([0.0, 90.0]))
    root = str(tmp_path)
    C.write_case(case, root)
    O.run_case(root)
    O.postproc(root)
    rd = os.path.join(root, "case", "results")
    F = G.decode_forces(case, np.loadtxt(os.path.join(rd, "Forces.dat"), ndmin=2))   # (nint, npb, nw)
    nb_, nr, nw, nint = len(case.betas_deg), len(case.rad), len(case.omegas), len(case.force)
    rc = open(os.path.join(rd, "RadiationCoefficients.tec")).read().split("\n")
    assert rc[0] == 'VARIABLES="w (rad/s)"' and rc[1] == '"A   1   1" "B   1   1"'
    assert rc[1 + nint] == 'Zone t="Motion of body    1 in DoF   1",I=     3,F=POINT'
    rows = np.array([[float(v) for v in l.split()] for l in rc[2 + nint:2 + nint + nw]])
    for iw, w in enumerate(case.omegas):
        assert rows[iw, 0] == w
        # A = Im(F)/w, B = -Re(F) of the surge radiation problem, per force
        np.testing.assert_allclose(rows[iw, 1::2], F[:, nb_, iw].imag / w, rtol=1e-15, atol=0)
        np.testing.assert_allclose(rows[iw, 2::2], -F[:, nb_, iw].real, rtol=1e-15, atol=0)
    fk = C.froude_krylov(case)   # (nw, nbeta, nint)
    ex = open(os.path.join(rd, "ExcitationForce.tec")).read().split("\n")
    zone = [i for i, l in enumerate(ex) if l.startswith("Zone")][1]
    assert ex[zone] == 'Zone t="Diffraction force - beta =  90.000 deg",I=     3,F=POINT'
    rows = np.array([[float(v) for v in l.split()] for l in ex[zone + 1:zone + 1 + nw]])
    tot = F[:, 1, :].T + fk[:, 1, :]
    np.testing.assert_allclose(rows[:, 1::2], np.abs(tot), rtol=1e-12)
    ca = open(os.path.join(rd, "CA.dat")).read().split("\n")
    assert ca[0] == "Nb de periode :     3"
    irf = open(os.path.join(rd, "IRF.tec")).read().split("\n")
    assert irf[0] == ' VARIABLES="Time (s)"' and irf[1 + nint] == 'Zone t="DoF    1",I=    20,F=POINT'
    for name in ("DiffractionForce.tec", "CM.dat", "Fe.dat"):
        assert os.path.getsize(os.path.join(rd, name)) > 0
