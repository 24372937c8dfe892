"""Extract the reference's own verification data into small JSON fixtures.

Nemoh ships three solver verification cases under Verification/ (a symmetric
vertical cylinder in deep water, a non-symmetric body in deep water, and two
bodies in 20 m finite depth), each with the mesh files, Nemoh.cal and reference
results (results/Aquaplus/Cw.tec: damping CA and added mass CM per DOF pair
over 150 frequencies; Fex.tec: excitation force magnitude and phase by wave
period). This script reads them from a Nemoh source tree and writes, per case,
the mesh, environment, DOFs and the reference coefficients at a subset of
frequencies, so that the tests can run without the source tree.

A fourth case, Verification/Postprocessing (the rotated cube of 2Bodies alone in
10 m of water, diffraction at omega = 0.8 rad/s, heading 0), ships the
free-surface elevation on the pre-processor's 50 x 50 grid over 400 m x 400 m
(Results/Aquaplus/FS.tec, zone "SUR LI": x, y, z, Re, Im, modulus) and the Kochin
function every 5 degrees (Results/Aquaplus/ZKochin.tec: theta, modulus, phase in
degrees). Every fifth grid point, the 24 points nearest the body, and every
direction are kept.

Usage: python tests/golden/make_verification_fixtures.py <nemoh-tree>
"""
import json
import os
import re
import sys

import numpy as np

CASES = {
    # name: (results dir, frequency stride into the 150-point table, max count)
    "Cylinder": ("results", 15, 10),
    "NonSymmetrical": ("Results", 15, 10),
    "2Bodies": ("Results", 15, 10),
}


def read_body(path):
    lines = open(path).read().split("\n")
    isym = int(lines[0].split()[1])
    nodes, i = [], 1
    while True:
        t = lines[i].split()
        i += 1
        if int(t[0]) == 0:
            break
        nodes.append([float(v) for v in t[1:4]])
    panels = []
    while True:
        t = lines[i].split()
        i += 1
        if int(t[0]) == 0:
            break
        panels.append([int(v) for v in t[:4]])
    return isym, nodes, panels


def parse_cal(d):
    L = [l.split("!")[0].split() for l in open(os.path.join(d, "Nemoh.cal")).read().split("\n")]
    out = {"rho": float(L[1][0]), "g": float(L[2][0]), "depth": float(L[3][0]), "bodies": []}
    nb = int(L[6][0])
    i = 7
    for b in range(1, nb + 1):
        i += 1
        fname = L[i][0]
        i += 2
        body = {"mesh_file": fname, "rad": [], "force": []}
        for key in ("rad", "force"):
            n = int(L[i][0])
            i += 1
            for _ in range(n):
                t = L[i]
                body[key].append([int(t[0])] + [float(v) for v in t[1:7]])
                i += 1
        na = int(L[i][0])
        i += 1 + na
        isym, nodes, panels = read_body(os.path.join(d, fname))
        body.update(isym=isym, nodes=nodes, panels=panels)
        out["bodies"].append(body)
    i += 2
    t = L[i]
    nbeta, bmin, bmax = int(t[0]), float(t[1]), float(t[2])
    out["betas_deg"] = list(np.linspace(bmin, bmax, nbeta)) if nbeta > 1 else [bmin]
    return out


def read_cw(path):
    zones = {}
    for blk in open(path).read().split("Zone")[1:]:
        hdr, body = blk.split("\n", 1)
        m = re.search(r"sur\s+(\d+)-\s*Mvt de\s+(\d+)\s+(\d)(\d)", hdr)
        arr = [[float(v) for v in l.split()] for l in body.strip().split("\n") if l.strip()]
        zones["%s,%s,%s,%s" % m.groups()] = arr
    return zones


def read_fex(path):
    nums = []
    for l in open(path).read().split("\n")[3:]:
        for t in l.split():
            try:
                nums.append(float(t))
            except ValueError:
                pass
    return np.array(nums)


def main(tree):
    here = os.path.dirname(os.path.abspath(__file__))
    for name, (rd, stride, count) in CASES.items():
        d = os.path.join(tree, "Verification", name)
        fx = parse_cal(d)
        zones = read_cw(os.path.join(d, rd, "Aquaplus", "Cw.tec"))
        w_all = np.array(next(iter(zones.values())))[:, 0]
        idx = list(range(0, len(w_all), stride))[:count]
        fx["omegas"] = [float(w_all[i]) for i in idx]
        # CA (damping), CM (added mass) at the selected omegas, plus the family
        # maxima over all 150 frequencies (used to scale the comparison)
        fx["cw"] = {}
        for k, arr in zones.items():
            a = np.array(arr)
            fx["cw"][k] = {"ca": [float(a[i, 1]) for i in idx], "cm": [float(a[i, 2]) for i in idx],
                           "ca_max": float(np.abs(a[:, 1]).max()), "cm_max": float(np.abs(a[:, 2]).max())}
        nums = read_fex(os.path.join(d, rd, "Aquaplus", "Fex.tec"))
        nf = 1 + 12 * len(fx["bodies"])
        if nums.size % nf == 0:
            A = nums.reshape(-1, nf)
            sel = list(range(0, len(A), max(1, len(A) // 8)))[:8]
            fx["fex"] = {"omega": [float(2 * np.pi / A[i, 0]) for i in sel],
                         "mag": [[float(v) for v in A[i, 1:1 + 6 * len(fx["bodies"])]] for i in sel]}
        out = os.path.join(here, "verification_%s.json" % name)
        with open(out, "w") as f:
            json.dump(fx, f)
        print("wrote", out, os.path.getsize(out), "bytes")
    postprocessing(tree, here)


def postprocessing(tree, here):
    d = os.path.join(tree, "Verification", "Postprocessing")
    fx = parse_cal(d)
    L = [l.split("!")[0].split() for l in open(os.path.join(d, "Nemoh.cal")).read().split("\n")]
    i = [n for n, l in enumerate(L) if l and l[0] == "---" and "Load" in " ".join(l)][0]
    nw, wmin, wmax = int(L[i + 1][0]), float(L[i + 1][1]), float(L[i + 1][2])
    fx["omegas"] = list(np.linspace(wmin, wmax, nw)) if nw > 1 else [wmin]
    fx["fs_grid"] = [int(L[i + 7][0]), int(L[i + 7][1]), float(L[i + 7][2]), float(L[i + 7][3])]
    lines = open(os.path.join(d, "Results", "Aquaplus", "FS.tec")).read().split("\n")
    z = [n for n, l in enumerate(lines) if "SUR LI" in l][0]
    npts = int(re.search(r"I=\s*(\d+)", lines[z]).group(1))
    A = np.array([[float(v) for v in l.split()] for l in lines[z + 1:z + 1 + npts]])
    r = np.hypot(A[:, 0], A[:, 1])
    keep = sorted(set(range(0, npts, 5)) | set(np.argsort(r)[:24].tolist()))
    fx["freesurface"] = {"index": keep, "x": A[keep, 0].tolist(), "y": A[keep, 1].tolist(),
                         "re": A[keep, 3].tolist(), "im": A[keep, 4].tolist()}
    K = np.loadtxt(os.path.join(d, "Results", "Aquaplus", "ZKochin.tec"), skiprows=1)
    fx["kochin"] = {"theta_deg": K[:, 0].tolist(), "abs": K[:, 1].tolist(), "arg_deg": K[:, 2].tolist()}
    out = os.path.join(here, "verification_Postprocessing.json")
    with open(out, "w") as f:
        json.dump(fx, f)
    print("wrote", out, os.path.getsize(out), "bytes")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_verification_fixtures.py <nemoh-source-tree>")
    main(sys.argv[1])
