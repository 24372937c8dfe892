"""Synthetic Nemoh cases, written in the reference Solver's own file formats.

This module plays the part of Nemoh's pre-processor for the synthetic
workloads: it builds panel meshes (vertical cylinder, rectangular barge,
hemispheres, boxes), computes the pre-processor's panel quantities
(preProcessor/Mesh.f90:197-222), the radiation and diffraction body
conditions (preProcessor/BodyConditions.f90:27-137 with
Common/Environment.f90:45-100), the generalised normals
(preProcessor/Integration.f90:27-86) and the Froude-Krylov forces
(preProcessor/Main.f90:223-243), and writes a case directory that the
reference Solver (and this package's drop-in driver) reads unchanged:

    ID.dat, <case>/Nemoh.cal, <case>/input.txt,
    <case>/mesh/L10.dat, <case>/mesh/L12.dat (Common/Mesh.f90:81-132),
    <case>/Normalvelocities.dat (Solver/Core/Bodyconditions.f90:65-89),
    <case>/mesh/Integration.dat (Solver/NEMOH.f90:88-94),
    <case>/mesh/Kochin.dat, <case>/mesh/Freesurface.dat (NEMOH.f90:96-118),
    <case>/results/FKForce.dat, <case>/results/index.dat.

Reals are written with 17 significant digits so that a double round-trips
exactly (the reference writes E14.7, too short for an FP64 comparison).

Problem order follows preProcessor/Main.f90:223-243: omega-major, and for
each omega the diffraction headings first, then the radiation DOFs.
"""
from __future__ import annotations

import dataclasses
import math
import os
from typing import List, Optional, Sequence

import numpy as np

__all__ = [
    "Mesh", "Dof", "Case", "six_dofs",
    "cylinder_mesh", "box_mesh", "hemisphere_mesh", "icosphere_hull", "merge_meshes",
    "panel_quantities", "wavenumber", "body_conditions", "generalised_normals",
    "froude_krylov", "write_case", "read_case", "CaseArrays",
    "config_cylinder", "config_barge", "config_two_spheres",
    "random_body", "config_batch", "serving_stream",
]


# --------------------------------------------------------------------------
# data model
# --------------------------------------------------------------------------
@dataclasses.dataclass
class Mesh:
    """Panel mesh: nodes (NP,3) float64 and panels (N,4) 1-based node ids."""
    nodes: np.ndarray
    panels: np.ndarray
    isym: int = 0                       # 1: only the y>=0 half is meshed
    body: Optional[np.ndarray] = None   # (N,) 1-based body id of each panel
    nbodies: int = 1

    def __post_init__(self):
        self.nodes = np.ascontiguousarray(self.nodes, dtype=np.float64)
        self.panels = np.ascontiguousarray(self.panels, dtype=np.int32)
        if self.body is None:
            self.body = np.ones(len(self.panels), dtype=np.int32)

    @property
    def npoints(self) -> int:
        return int(self.nodes.shape[0])

    @property
    def npanels(self) -> int:
        return int(self.panels.shape[0])


@dataclasses.dataclass
class Dof:
    """One radiation DOF or force-integration case (Nemoh.cal body block).

    icase 1 = translation along `direction`; icase 2 = rotation about the
    axis through `axis` with direction `direction`.
    """
    icase: int
    direction: Sequence[float]
    axis: Sequence[float] = (0.0, 0.0, 0.0)
    body: int = 1


def six_dofs(center=(0.0, 0.0, 0.0), body: int = 1) -> List[Dof]:
    c = tuple(float(v) for v in center)
    return [Dof(1, (1, 0, 0), c, body), Dof(1, (0, 1, 0), c, body),
            Dof(1, (0, 0, 1), c, body), Dof(2, (1, 0, 0), c, body),
            Dof(2, (0, 1, 0), c, body), Dof(2, (0, 0, 1), c, body)]


@dataclasses.dataclass
class Case:
    mesh: Mesh
    omegas: np.ndarray
    betas_deg: np.ndarray
    rad: List[Dof]
    force: List[Dof]
    rho: float = 1025.0
    g: float = 9.81
    depth: float = 0.0
    xeff: float = 0.0
    yeff: float = 0.0
    name: str = "case"
    kochin_theta: tuple = ()   # directions (rad) of mesh/Kochin.dat; Kochin switch set for every problem if any
    fs_grid: tuple = ()        # (Nx, Ny, Lx, Ly) of Nemoh.cal's free-surface line; free-surface switch set if any
    irf: tuple = ()            # (dt, duration) of Nemoh.cal's IRF line; IRF switch set if given

    @property
    def nproblems(self) -> int:
        return len(self.omegas) * (len(self.betas_deg) + len(self.rad))


# --------------------------------------------------------------------------
# mesh builders
# --------------------------------------------------------------------------
class _NodeSet:
    """Deduplicating node table (1-based ids)."""

    def __init__(self):
        self.ids = {}
        self.xyz = []

    def add(self, p) -> int:
        key = tuple(int(round(v * 1e9)) for v in p)
        i = self.ids.get(key)
        if i is None:
            self.xyz.append([float(p[0]), float(p[1]), float(p[2])])
            i = len(self.xyz)
            self.ids[key] = i
        return i


def _orient(nodes: np.ndarray, panels: np.ndarray, centers: np.ndarray) -> np.ndarray:
    """Reverse panels whose normal points into the body (convex bodies).

    The Solver's normal is (P3-P1)x(P4-P2) (Solver/Core/PREPARE_MESH.f90:96-107)
    and must point out of the body, into the fluid.
    """
    p = panels - 1
    t1 = nodes[p[:, 2]] - nodes[p[:, 0]]
    t2 = nodes[p[:, 3]] - nodes[p[:, 1]]
    n = np.cross(t1, t2)
    xm = nodes[p].mean(axis=1)
    bad = np.einsum("ij,ij->i", n, xm - centers) < 0
    out = panels.copy()
    out[bad] = out[bad][:, [0, 3, 2, 1]]
    return out


def cylinder_mesh(radius=5.0, draft=10.0, n_theta=24, n_z=10, n_rings=5,
                  n_sectors=12, half=False, center=(0.0, 0.0)) -> Mesh:
    """Truncated vertical cylinder: side wall plus a flat bottom disc.

    The bottom's innermost ring is made of quads with a repeated centre node
    (triangles), as Nemoh meshes commonly are. `half` meshes only y>=0 (Isym=1).
    """
    cx, cy = center
    ns = _NodeSet()
    quads = []
    tmax = math.pi if half else 2.0 * math.pi
    nth = n_theta // 2 if half else n_theta
    ths = [tmax * k / nth for k in range(nth + 1)]
    zs = [-draft + draft * l / n_z for l in range(n_z + 1)]

    def side(k, l):
        return ns.add((cx + radius * math.cos(ths[k]), cy + radius * math.sin(ths[k]), zs[l]))

    for k in range(nth):
        for l in range(n_z):
            quads.append([side(k + 1, l), side(k + 1, l + 1), side(k, l + 1), side(k, l)])
    nsec = n_sectors // 2 if half else n_sectors
    phs = [tmax * s / nsec for s in range(nsec + 1)]
    rs = [radius * i / n_rings for i in range(n_rings + 1)]

    def bot(i, s):
        if i == 0:
            return ns.add((cx, cy, -draft))
        return ns.add((cx + rs[i] * math.cos(phs[s]), cy + rs[i] * math.sin(phs[s]), -draft))

    for i in range(n_rings):
        for s in range(nsec):
            quads.append([bot(i, s), bot(i, s + 1), bot(i + 1, s + 1), bot(i + 1, s)])
    nodes = np.array(ns.xyz)
    panels = np.array(quads, dtype=np.int32)
    cen = np.tile([cx, cy, -draft / 2.0], (len(panels), 1))
    return Mesh(nodes, _orient(nodes, panels, cen), isym=1 if half else 0)


def box_mesh(length=100.0, beam=20.0, draft=10.0, nx=50, ny=20, nz=20,
             half=False, center=(0.0, 0.0)) -> Mesh:
    """Rectangular box (barge) with its deck at z=0.

    nx, ny, nz are panel counts along the length, the (half) beam and the
    draft. With `half`, only y>=0 is meshed and ny spans beam/2.
    """
    cx, cy = center
    ns = _NodeSet()
    quads = []
    x0, x1 = cx - length / 2, cx + length / 2
    y0 = cy if half else cy - beam / 2
    y1 = cy + beam / 2
    xs = np.linspace(x0, x1, nx + 1)
    ys = np.linspace(y0, y1, ny + 1)
    zs = np.linspace(-draft, 0.0, nz + 1)

    def grid(a, b, fn):
        for i in range(len(a) - 1):
            for j in range(len(b) - 1):
                quads.append([ns.add(fn(a[i], b[j])), ns.add(fn(a[i + 1], b[j])),
                              ns.add(fn(a[i + 1], b[j + 1])), ns.add(fn(a[i], b[j + 1]))])

    grid(xs, zs, lambda x, z: (x, y1, z))            # side y = +beam/2
    if not half:
        grid(xs, zs, lambda x, z: (x, y0, z))        # side y = -beam/2
    grid(xs, ys, lambda x, y: (x, y, -draft))        # bottom
    grid(ys, zs, lambda y, z: (x0, y, z))            # end x = x0
    grid(ys, zs, lambda y, z: (x1, y, z))            # end x = x1
    nodes = np.array(ns.xyz)
    panels = np.array(quads, dtype=np.int32)
    cen = np.tile([cx, cy, -draft / 2.0], (len(panels), 1))
    return Mesh(nodes, _orient(nodes, panels, cen), isym=1 if half else 0)


def hemisphere_mesh(radius=4.0, n_lat=40, n_lon=100, center=(0.0, 0.0),
                    draft=None, half=False, jitter=0.0, rng=None) -> Mesh:
    """Submerged part of a floating sphere, latitude-longitude panels.

    `draft` (<= radius) sets how deep the sphere's lowest point sits; the
    sphere centre is at z = radius - draft (default: half submerged). The
    last band at the bottom pole holds triangles (repeated pole node).
    `jitter` moves interior nodes tangentially by that fraction of the local
    spacing (seeded by `rng`), which spreads panel areas.
    """
    cx, cy = center
    if draft is None:
        draft = radius
    zc = radius - draft
    # polar angle from the bottom pole (0) up to the waterline
    phi_w = math.acos(max(-1.0, min(1.0, zc / radius)))  # bottom pole to waterline
    lon_max = math.pi if half else 2.0 * math.pi
    nlon = n_lon // 2 if half else n_lon
    ns = _NodeSet()
    pts = {}
    # equal-area latitude bands: cos(a) uniformly spaced (Archimedes)
    cw = math.cos(phi_w)
    alat = [math.acos(max(-1.0, min(1.0, 1.0 - (1.0 - cw) * i / n_lat))) for i in range(n_lat + 1)]
    for i in range(n_lat + 1):
        a = alat[i]
        for j in range(nlon + 1):
            b = lon_max * j / nlon
            if not half and j == nlon:
                pts[(i, j)] = pts[(i, 0)]
                continue
            if i == 0:
                p = (cx, cy, zc - radius)
            else:
                r = radius * math.sin(a)
                p = [cx + r * math.cos(b), cy + r * math.sin(b), zc - radius * math.cos(a)]
                interior = 0 < i < n_lat and (not half or 0 < j < nlon)
                if jitter and interior and rng is not None:
                    da = 0.5 * (alat[i + 1] - alat[i - 1]) * jitter * rng.uniform(-1, 1)
                    db = lon_max / nlon * jitter * rng.uniform(-1, 1)
                    a2, b2 = a + da, b + db
                    r2 = radius * math.sin(a2)
                    p = [cx + r2 * math.cos(b2), cy + r2 * math.sin(b2), zc - radius * math.cos(a2)]
                if i == n_lat:
                    p[2] = 0.0 if abs(p[2]) < 1e-12 else p[2]
            pts[(i, j)] = ns.add(p)
    quads = []
    for i in range(n_lat):
        for j in range(nlon):
            quads.append([pts[(i, j)], pts[(i, j + 1)], pts[(i + 1, j + 1)], pts[(i + 1, j)]])
    nodes = np.array(ns.xyz)
    panels = np.array(quads, dtype=np.int32)
    cen = np.tile([cx, cy, zc], (len(panels), 1))
    return Mesh(nodes, _orient(nodes, panels, cen), isym=1 if half else 0)


_ICO_FACES = ((0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2),
              (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5), (2, 4, 11),
              (6, 2, 10), (8, 6, 7), (9, 8, 1))


def _icosahedron():
    t = (1.0 + 5.0 ** 0.5) / 2.0
    v = np.array([[-1, t, 0], [1, t, 0], [-1, -t, 0], [1, -t, 0], [0, -1, t], [0, 1, t], [0, -1, -t], [0, 1, -t],
                  [t, 0, -1], [t, 0, 1], [-t, 0, -1], [-t, 0, 1]], dtype=np.float64)
    return v / np.linalg.norm(v, axis=1)[:, None]


def icosphere_hull(radius=4.0, freq=12, cut=-0.055, center=(0.0, 0.0), n_target=None, jitter=0.0, rng=None) -> Mesh:
    """Submerged part of a floating sphere from a geodesic icosphere, in quads.

    The icosahedron's faces are subdivided into freq^2 triangles each and
    projected on the unit sphere; the triangles whose centroid lies below
    z = cut (in sphere radii) are kept and their vertices above the plane are
    levelled onto it (moved down the sphere to the waterline circle). Each
    triangle is split into three quads (vertex, two edge midpoints and the
    centroid, projected on the sphere; waterline midpoints stay on the
    waterline). With `n_target`, the largest quads are halved (across their
    longer pair of opposite edges) until that count is reached. The sphere is
    then scaled to `radius` and placed so that the waterline is z = 0 at
    `center`. `jitter` moves every node off the waterline tangentially by up
    to that fraction of the local edge length (seeded by `rng`), which changes
    panel areas by up to about the same fraction.
    """
    V = _icosahedron()
    ns = _NodeSet()
    zc = math.sqrt(max(0.0, 1.0 - cut * cut))

    def level(p):
        p = p / np.linalg.norm(p)
        if p[2] > cut:   # onto the waterline circle, same azimuth
            r = math.hypot(p[0], p[1])
            p = np.array([p[0] * zc / r, p[1] * zc / r, cut])
        return p

    tris = []
    for a, b, c in _ICO_FACES:
        A, B, Cc = V[a], V[b], V[c]
        P = {}
        for i in range(freq + 1):
            for j in range(freq + 1 - i):
                p = A + (B - A) * i / freq + (Cc - A) * j / freq
                P[(i, j)] = p / np.linalg.norm(p)
        for i in range(freq):
            for j in range(freq - i):
                tris.append((P[(i, j)], P[(i + 1, j)], P[(i, j + 1)]))
                if i + j + 1 < freq:
                    tris.append((P[(i + 1, j)], P[(i + 1, j + 1)], P[(i, j + 1)]))
    kept = [tuple(level(v) for v in t) for t in tris if (t[0][2] + t[1][2] + t[2][2]) / 3.0 < cut]

    def mid(p, q):
        m = 0.5 * (p + q)
        if abs(p[2] - cut) < 1e-12 and abs(q[2] - cut) < 1e-12:   # a waterline edge
            r = math.hypot(m[0], m[1])
            return np.array([m[0] * zc / r, m[1] * zc / r, cut])
        return m / np.linalg.norm(m)

    quads = []
    for v0, v1, v2 in kept:
        c = (v0 + v1 + v2) / np.linalg.norm(v0 + v1 + v2)
        m01, m12, m20 = mid(v0, v1), mid(v1, v2), mid(v2, v0)
        quads += [[v0, m01, c, m20], [v1, m12, c, m01], [v2, m20, c, m12]]

    def quad_area(q):
        return 0.5 * np.linalg.norm(np.cross(q[2] - q[0], q[3] - q[1]))

    if n_target is not None:
        if n_target < len(quads):
            raise ValueError("icosphere_hull: %d quads exceed the target %d" % (len(quads), n_target))
        while len(quads) < n_target:
            k = max(range(len(quads)), key=lambda i: quad_area(quads[i]))
            p0, p1, p2, p3 = quads.pop(k)
            if np.linalg.norm(p1 - p0) + np.linalg.norm(p3 - p2) >= np.linalg.norm(p2 - p1) + np.linalg.norm(p0 - p3):
                a, b = mid(p0, p1), mid(p2, p3)       # halve edges p0p1 and p2p3
                quads += [[p0, a, b, p3], [a, p1, p2, b]]
            else:
                a, b = mid(p1, p2), mid(p3, p0)       # halve edges p1p2 and p3p0
                quads += [[p0, p1, a, b], [b, a, p2, p3]]
    ids = [[ns.add(tuple(v)) for v in q] for q in quads]
    nodes = np.array(ns.xyz)
    if jitter and rng is not None:
        panels0 = np.array(ids) - 1
        edge = np.zeros(len(nodes))
        cnt = np.zeros(len(nodes))
        for q in panels0:
            for k in range(4):
                a, b = q[k], q[(k + 1) % 4]
                d = np.linalg.norm(nodes[a] - nodes[b])
                edge[a] += d
                edge[b] += d
                cnt[a] += 1
                cnt[b] += 1
        h = edge / np.maximum(cnt, 1)
        for i in range(len(nodes)):
            p = nodes[i]
            if abs(p[2] - cut) < 1e-12:
                continue   # the waterline stays in the plane
            t1 = np.cross(p, [0.0, 0.0, 1.0] if abs(p[2]) < 0.9 else [1.0, 0.0, 0.0])
            t1 /= np.linalg.norm(t1)
            t2 = np.cross(p, t1)
            d = jitter * h[i] * rng.uniform(-1, 1, 2)
            q = p + d[0] * t1 + d[1] * t2
            q /= np.linalg.norm(q)
            nodes[i] = q if q[2] < cut else p
    nodes = nodes * radius
    nodes[:, 2] -= cut * radius
    nodes[:, 0] += center[0]
    nodes[:, 1] += center[1]
    panels = np.array(ids, dtype=np.int32)
    cen = np.tile([center[0], center[1], -cut * radius], (len(panels), 1))
    return Mesh(nodes, _orient(nodes, panels, cen), isym=0)


def merge_meshes(meshes: Sequence[Mesh]) -> Mesh:
    """Concatenate bodies into one multi-body mesh (body ids 1..n)."""
    nodes, panels, body = [], [], []
    off = 0
    for b, m in enumerate(meshes):
        nodes.append(m.nodes)
        panels.append(m.panels + off)
        body.append(np.full(m.npanels, b + 1, dtype=np.int32))
        off += m.npoints
    isym = meshes[0].isym
    assert all(m.isym == isym for m in meshes)
    return Mesh(np.vstack(nodes), np.vstack(panels), isym, np.concatenate(body), len(meshes))


# --------------------------------------------------------------------------
# pre-processor quantities
# --------------------------------------------------------------------------
def panel_quantities(mesh: Mesh):
    """(XM (N,3), normal (N,3), area (N,)) as preProcessor/Mesh.f90:197-222."""
    x = mesh.nodes
    p = mesh.panels - 1
    w1 = np.cross(x[p[:, 1]] - x[p[:, 0]], x[p[:, 3]] - x[p[:, 1]])
    a1 = 0.5 * np.linalg.norm(w1, axis=1)
    w2 = np.cross(x[p[:, 3]] - x[p[:, 2]], x[p[:, 1]] - x[p[:, 2]])
    a2 = 0.5 * np.linalg.norm(w2, axis=1)
    a = a1 + a2
    if np.any(a < 1.0e-7):
        raise ValueError("panel area below 1e-7 (preProcessor/Mesh.f90:206-209)")
    xm = ((1.0 / 3) * (x[p[:, 0]] + x[p[:, 1]] + x[p[:, 3]]) * (a1 / a)[:, None]
          + (1.0 / 3) * (x[p[:, 1]] + x[p[:, 2]] + x[p[:, 3]]) * (a2 / a)[:, None])
    u = w1 + w2
    n = u / np.linalg.norm(u, axis=1)[:, None]
    return xm, n, a


def wavenumber(w: float, g: float, depth: float) -> float:
    """Common/Environment.f90:45-85 (bisection to 1e-6 on x tanh x = w^2 h/g)."""
    k = w * w / g
    x0 = k * depth
    if 0.0 < x0 <= 20.0:
        xg, xd = 0.0, x0
        nite = 0
        while nite < 10000 and (x0 - xg * math.tanh(xg)) * (x0 - xd * math.tanh(xd)) > 0.0:
            xg, xd = xd, 2.0 * xd
            nite += 1
        nite = 0
        xc = 0.5 * (xd + xg)
        while nite < 10000 and abs(xd - xg) / abs(xc) >= 1.0e-6:
            xc = 0.5 * (xd + xg)
            if (x0 - xg * math.tanh(xg)) * (x0 - xc * math.tanh(xc)) > 0.0:
                xg = xc
            else:
                xd = xc
            nite += 1
        k = xc / depth
    return k


def _cih(k, z, h):
    if k * h <= 20 and k * h > 0.0:
        return np.cosh(k * (z + h)) / math.cosh(k * h)
    return np.exp(k * z)


def _sih(k, z, h):
    if k * h <= 20 and k * h > 0.0:
        return np.sinh(k * (z + h)) / math.cosh(k * h)
    return np.exp(k * z)


def _wave(case: Case, k, w, beta, x, y, z):
    """Compute_Wave (Common/Environment.f90:86-100) vectorised over points."""
    g = case.g
    wbar = (x - case.xeff) * math.cos(beta) + (y - case.yeff) * math.sin(beta)
    e = np.exp(1j * k * wbar)
    cih = _cih(k, z, case.depth)
    sih = _sih(k, z, case.depth)
    p = case.rho * g * cih * e
    vx = g / w * k * math.cos(beta) * cih * e
    vy = g / w * k * math.sin(beta) * cih * e
    vz = -1j * g / w * k * sih * e
    return p, vx, vy, vz


def _dof_vector(mesh: Mesh, xm, n, a, dof: Dof, scale_area: bool):
    """Radiation normal velocity / NDS for one DOF, both halves if Isym=1."""
    sel = (mesh.body == dof.body).astype(np.float64)
    d = np.asarray(dof.direction, dtype=np.float64)
    ax = np.asarray(dof.axis, dtype=np.float64)
    area = a if scale_area else np.ones_like(a)
    halves = [(xm, n)]
    if mesh.isym == 1:
        xm2 = xm.copy()
        xm2[:, 1] = -xm2[:, 1]
        n2 = n.copy()
        n2[:, 1] = -n2[:, 1]
        halves.append((xm2, n2))
    out = []
    for xh, nh in halves:
        if dof.icase == 1:
            vel = np.tile(d, (len(xh), 1))
        elif dof.icase == 2:
            vel = np.cross(d, xh - ax)
        else:
            raise ValueError("unknown DOF case %d" % dof.icase)
        out.append(np.einsum("ij,ij->i", nh, vel) * area * sel)
    return np.concatenate(out)


def body_conditions(case: Case):
    """NVEL (2^s*N, Nproblems) complex, in the pre-processor's problem order."""
    mesh = case.mesh
    xm, n, a = panel_quantities(mesh)
    nb, nr = len(case.betas_deg), len(case.rad)
    out = np.zeros((mesh.npanels * 2 ** mesh.isym, case.nproblems), dtype=np.complex128)
    rad = [_dof_vector(mesh, xm, n, a, d, False) for d in case.rad]
    for i, w in enumerate(case.omegas):
        k = wavenumber(float(w), case.g, case.depth)
        for j, bdeg in enumerate(case.betas_deg):
            beta = bdeg * math.pi / 180.0
            cols = []
            _, vx, vy, vz = _wave(case, k, w, beta, xm[:, 0], xm[:, 1], xm[:, 2])
            cols.append(-(vx * n[:, 0] + vy * n[:, 1] + vz * n[:, 2]))
            if mesh.isym == 1:
                _, vx, vy, vz = _wave(case, k, w, beta, xm[:, 0], -xm[:, 1], xm[:, 2])
                cols.append(-(vx * n[:, 0] - vy * n[:, 1] + vz * n[:, 2]))
            out[:, j + i * (nb + nr)] = np.concatenate(cols)
        for j in range(nr):
            out[:, nb + j + i * (nb + nr)] = rad[j]
    return out


def generalised_normals(case: Case):
    """NDS (Nint, 2^s*N) real, preProcessor/Integration.f90:27-86."""
    xm, n, a = panel_quantities(case.mesh)
    return np.stack([_dof_vector(case.mesh, xm, n, a, d, True) for d in case.force])


def froude_krylov(case: Case):
    """FK force (Nw, Nbeta, Nint) complex, preProcessor/Main.f90:223-235."""
    mesh = case.mesh
    xm, n, a = panel_quantities(mesh)
    nds = generalised_normals(case)
    out = np.zeros((len(case.omegas), len(case.betas_deg), len(case.force)), dtype=np.complex128)
    for i, w in enumerate(case.omegas):
        k = wavenumber(float(w), case.g, case.depth)
        for j, bdeg in enumerate(case.betas_deg):
            beta = bdeg * math.pi / 180.0
            p, *_ = _wave(case, k, w, beta, xm[:, 0], xm[:, 1], xm[:, 2])
            if mesh.isym == 1:
                p2, *_ = _wave(case, k, w, beta, xm[:, 0], -xm[:, 1], xm[:, 2])
                p = np.concatenate([p, p2])
            out[i, j, :] = -(nds * p[None, :]).sum(axis=1)
    return out


# --------------------------------------------------------------------------
# writers / readers of the reference formats
# --------------------------------------------------------------------------
def _r(v) -> str:
    return repr(float(v))


def freesurface_grid(nx, ny, lx, ly):
    """Free-surface visualisation grid of the pre-processor (preProcessor/Main.f90:287-300):
    nx * ny points (x, y) on an lx by ly rectangle centred on the origin, x
    outer and y inner, and the (nx-1)(ny-1) quadrangles as 1-based point numbers."""
    nx, ny = int(nx), int(ny)
    pts = [(-0.5 * lx + lx * i / (nx - 1), -0.5 * ly + ly * j / (ny - 1)) for i in range(nx) for j in range(ny)]
    quads = [(j + 1 + i * ny, j + 2 + i * ny, j + 2 + (i + 1) * ny, j + 1 + (i + 1) * ny)
             for i in range(nx - 1) for j in range(ny - 1)]
    return np.array(pts), np.array(quads, dtype=np.int64).reshape(-1, 4)


def write_case(case: Case, root: str, case_dir: str = "case") -> str:
    """Write ID.dat in `root` and the case directory `root/case_dir`."""
    mesh = case.mesh
    d = os.path.join(root, case_dir)
    os.makedirs(os.path.join(d, "mesh"), exist_ok=True)
    os.makedirs(os.path.join(d, "results"), exist_ok=True)
    with open(os.path.join(root, "ID.dat"), "w") as f:
        f.write("%d\n%s\n" % (len(case_dir), case_dir))
    nb = mesh.nbodies
    with open(os.path.join(d, "Nemoh.cal"), "w") as f:
        f.write("--- Environment ---\n")
        f.write("%s\t! RHO\n%s\t! G\n%s\t! DEPTH\n%s %s\t! XEFF YEFF\n"
                % (_r(case.rho), _r(case.g), _r(case.depth), _r(case.xeff), _r(case.yeff)))
        f.write("--- Description of floating bodies ---\n%d\t! Number of bodies\n" % nb)
        for b in range(1, nb + 1):
            rad = [r for r in case.rad if r.body == b]
            frc = [r for r in case.force if r.body == b]
            npan = int((mesh.body == b).sum())
            f.write("--- Body %d ---\nbody%d.dat\n%d %d\n" % (b, b, mesh.npoints, npan))
            f.write("%d\n" % len(rad))
            for r in rad:
                f.write("%d %s %s %s %s %s %s\n" % ((r.icase,) + tuple(_r(v) for v in r.direction)
                                                    + tuple(_r(v) for v in r.axis)))
            f.write("%d\n" % len(frc))
            for r in frc:
                f.write("%d %s %s %s %s %s %s\n" % ((r.icase,) + tuple(_r(v) for v in r.direction)
                                                    + tuple(_r(v) for v in r.axis)))
            f.write("0\n")
        f.write("--- Load cases to be solved ---\n")
        om = case.omegas
        f.write("%d %s %s\n" % (len(om), _r(om[0]), _r(om[-1])))
        bt = case.betas_deg
        f.write("%d %s %s\n" % (len(bt), _r(bt[0]) if len(bt) else "0.", _r(bt[-1]) if len(bt) else "0."))
        kt = np.degrees(np.asarray(case.kochin_theta, dtype=float))
        fsg = tuple(case.fs_grid) if len(case.fs_grid) else (0, 0, 100.0, 100.0)
        irf = ("1 %s %s" % (_r(case.irf[0]), _r(case.irf[1]))) if len(case.irf) else "0 0.1 10."
        f.write("--- Post processing ---\n%s\n0\n%d %s %s\n%d %d %s %s\n"
                % (irf, len(kt), _r(kt[0]) if len(kt) else "0.", _r(kt[-1]) if len(kt) else "180.",
                   int(fsg[0]), int(fsg[1]), _r(fsg[2]), _r(fsg[3])))
    with open(os.path.join(d, "input.txt"), "w") as f:
        f.write("--- Calculation parameters ---\n0\n")
    # L12: "2 Isym", nodes, 0-line, panels, 0-line (Common/Mesh.f90:102-118)
    with open(os.path.join(d, "mesh", "L12.dat"), "w") as f:
        f.write("2 %d\n" % mesh.isym)
        for i, p in enumerate(mesh.nodes):
            f.write("%d %s %s %s\n" % (i + 1, _r(p[0]), _r(p[1]), _r(p[2])))
        f.write("0 0. 0. 0.\n")
        for q in mesh.panels:
            f.write("%d %d %d %d\n" % tuple(q))
        f.write("0 0 0 0\n")
    xm, n, a = panel_quantities(mesh)
    with open(os.path.join(d, "mesh", "L10.dat"), "w") as f:
        f.write("\n%d %d %d %d\n" % (mesh.isym, mesh.npoints, mesh.npanels, nb))
        for i in range(mesh.npanels):
            f.write("%d %s %s %s %s %s %s %s\n" % ((int(mesh.body[i]),) + tuple(_r(v) for v in xm[i])
                                                   + tuple(_r(v) for v in n[i]) + (_r(a[i]),)))
        f.write("0\n")
    nds = generalised_normals(case)
    with open(os.path.join(d, "mesh", "Integration.dat"), "w") as f:
        f.write("%d\n" % len(nds))
        for row in nds:
            f.write(" ".join(_r(v) for v in row) + "\n")
    nvel = body_conditions(case)
    nb_, nr = len(case.betas_deg), len(case.rad)
    npb = nb_ + nr
    with open(os.path.join(d, "Normalvelocities.dat"), "w") as f:
        f.write("%d\n" % case.nproblems)
        f.write(" ".join(_r(w) for w in case.omegas for _ in range(npb)) + "\n")
        for _ in case.omegas:
            f.write(" ".join([_r(b * math.pi / 180.0) for b in case.betas_deg] + ["-1.0"] * nr) + "\n")
        f.write(" ".join("0" for _ in range(case.nproblems)) + "\n")
        sfs = "1" if len(case.fs_grid) and case.fs_grid[0] > 0 else "0"
        f.write(" ".join(sfs for _ in range(case.nproblems)) + "\n")
        sk = "1" if len(case.kochin_theta) else "0"
        f.write(" ".join(sk for _ in range(case.nproblems)) + "\n")
        for c in range(nvel.shape[0]):
            f.write(" ".join("%s %s" % (_r(v.real), _r(v.imag)) for v in nvel[c]) + "\n")
    with open(os.path.join(d, "mesh", "Kochin.dat"), "w") as f:
        f.write("%d\n" % len(case.kochin_theta))
        for t in case.kochin_theta:
            f.write("%s\n" % _r(t))
    with open(os.path.join(d, "mesh", "Freesurface.dat"), "w") as f:
        if len(case.fs_grid) and case.fs_grid[0] > 0:
            pts, quads = freesurface_grid(*case.fs_grid)
            f.write("%d %d\n" % (len(pts), len(quads)))
            for x, y in pts:
                f.write("%s %s 0.\n" % (_r(x), _r(y)))
            for q in quads:
                f.write("%d %d %d %d\n" % tuple(q))
        else:
            f.write("0 0\n")
    fk = froude_krylov(case)
    with open(os.path.join(d, "results", "FKForce.dat"), "w") as f:
        for k in range(len(case.force)):
            vals = []
            for i in range(len(case.omegas)):
                for c in range(len(case.betas_deg)):
                    vals += [_r(abs(fk[i, c, k])), _r(math.atan2(fk[i, c, k].imag, fk[i, c, k].real))]
                vals += ["0.0", "0.0"] * nr
            f.write(" ".join(vals) + "\n")
    # FKForce.tec, the post-processor's source of Froude-Krylov forces
    # (preProcessor/Main.f90:266-276)
    with open(os.path.join(d, "results", "FKForce.tec"), "w") as f:
        f.write('VARIABLES="w (rad/s)"\n')
        for k, r in enumerate(case.force):
            f.write('"abs(F%4d%4d)" "angle(F%4d%4d)"\n' % (r.body, k + 1, r.body, k + 1))
        for c, b in enumerate(case.betas_deg):
            f.write('Zone t="FKforce - beta = %7.3f",I=%6d,F=POINT\n' % (b, len(case.omegas)))
            for i, w in enumerate(case.omegas):
                vals = [_r(w)]
                for k in range(len(case.force)):
                    vals += [_r(abs(fk[i, c, k])), _r(math.atan2(fk[i, c, k].imag, fk[i, c, k].real))]
                f.write(" ".join(vals) + "\n")

    def modes(dofs):   # index of each DOF within its body (Main.f90:160-176)
        seen = {}
        out = []
        for r in dofs:
            seen[r.body] = seen.get(r.body, 0) + 1
            out.append(seen[r.body])
        return out

    with open(os.path.join(d, "results", "index.dat"), "w") as f:
        f.write("%d %d %d %d %d\n" % (len(case.omegas), len(case.betas_deg), nr, len(case.force),
                                      len(case.kochin_theta)))
        f.write("--- Force ---\n")
        for k, (r, m) in enumerate(zip(case.force, modes(case.force))):
            f.write("%d %d %d\n" % (k + 1, r.body, m))
        f.write("--- Motion ---\n")
        for k, (r, m) in enumerate(zip(case.rad, modes(case.rad))):
            f.write("%d %d %d\n" % (k + 1, r.body, m))
        f.write(" ".join(_r(b * math.pi / 180.0) for b in case.betas_deg) + "\n")
        f.write(" ".join(_r(w) for w in case.omegas) + "\n")
        f.write(" ".join(_r(t) for t in case.kochin_theta) + "\n")
    return d


class _ListReader:
    """Fortran list-directed READ: each read starts a new record and may span lines."""

    def __init__(self, path):
        with open(path) as f:
            self.lines = f.read().splitlines()
        self.pos = 0

    def skip(self):
        self.pos += 1

    def read(self, n):
        vals = []
        while len(vals) < n:
            if self.pos >= len(self.lines):
                raise EOFError("unexpected end of file")
            line = self.lines[self.pos].split("!")[0]
            self.pos += 1
            toks = line.replace(",", " ").split()
            vals.extend(toks)
        return vals[:n]


@dataclasses.dataclass
class CaseArrays:
    """A case directory loaded into the arrays the Solver works on."""
    rho: float
    g: float
    depth: float
    isym: int
    nodes: np.ndarray        # (NP,3)
    panels: np.ndarray       # (N,4) 1-based
    omega: np.ndarray        # (Nproblems,)
    switch_type: np.ndarray  # (Nproblems,) beta in rad, or -1 for radiation
    nvel: np.ndarray         # (2^s N, Nproblems) complex
    nds: np.ndarray          # (Nint, 2^s N)


def read_case(root: str) -> CaseArrays:
    """Read ID.dat and the case files exactly as the reference Solver does."""
    r = _ListReader(os.path.join(root, "ID.dat"))
    lid = int(r.read(1)[0])
    cid = r.read(1)[0][:lid]
    d = os.path.join(root, cid)
    r = _ListReader(os.path.join(d, "mesh", "L10.dat"))
    r.skip()
    _, npts, npan, _ = (int(v) for v in r.read(4))
    r = _ListReader(os.path.join(d, "mesh", "L12.dat"))
    two, isym = (int(v) for v in r.read(2))
    if two != 2:
        raise ValueError("The mesh file format is not correct.")
    nodes = np.array([[float(v) for v in r.read(4)[1:]] for _ in range(npts)])
    r.skip()
    panels = np.array([[int(v) for v in r.read(4)] for _ in range(npan)], dtype=np.int32)
    r = _ListReader(os.path.join(d, "Nemoh.cal"))
    r.skip()
    rho = float(r.read(1)[0])
    g = float(r.read(1)[0])
    depth = float(r.read(1)[0])
    nc = npan * 2 ** isym
    r = _ListReader(os.path.join(d, "Normalvelocities.dat"))
    npb = int(r.read(1)[0])
    omega = np.array([float(v) for v in r.read(npb)])
    st = np.array([float(v) for v in r.read(npb)])
    for _ in range(3):
        r.read(npb)
    nvel = np.zeros((nc, npb), dtype=np.complex128)
    for c in range(nc):
        v = np.array([float(t) for t in r.read(2 * npb)])
        nvel[c] = v[0::2] + 1j * v[1::2]
    r = _ListReader(os.path.join(d, "mesh", "Integration.dat"))
    nint = int(r.read(1)[0])
    nds = np.array([[float(t) for t in r.read(nc)] for _ in range(nint)]).reshape(nint, nc)
    return CaseArrays(rho, g, depth, isym, nodes, panels, omega, st, nvel, nds)


# --------------------------------------------------------------------------
# the synthetic workloads
# --------------------------------------------------------------------------
def config_cylinder(n_omega=10) -> Case:
    """Truncated vertical cylinder R=5 m, draft 10 m, 300 panels, deep water."""
    mesh = cylinder_mesh(5.0, 10.0, 24, 10, 5, 12, half=False)
    return Case(mesh, np.linspace(0.1, 2.0, n_omega), np.array([0.0]),
                six_dofs(), six_dofs(), rho=1025.0, g=9.81, depth=0.0, name="cylinder300")


def config_barge(n_omega=40, nx=50, ny=20, nz=20, nye=10) -> Case:
    """Barge 100x20 m, draft 10 m, depth 50 m, y-symmetric half mesh.

    Default spacing gives 2,400 half-mesh panels: sides 50x20 (2 m x 0.5 m),
    bottom 50x20 (2 m x 0.5 m), two ends 10x20 (1 m x 0.5 m).
    """
    ns = _NodeSet()
    quads = []
    L, B, D = 100.0, 20.0, 10.0
    xs = np.linspace(-L / 2, L / 2, nx + 1)
    yb = np.linspace(0.0, B / 2, ny + 1)
    ye = np.linspace(0.0, B / 2, nye + 1)
    zs = np.linspace(-D, 0.0, nz + 1)

    def grid(a, b, fn):
        for i in range(len(a) - 1):
            for j in range(len(b) - 1):
                quads.append([ns.add(fn(a[i], b[j])), ns.add(fn(a[i + 1], b[j])),
                              ns.add(fn(a[i + 1], b[j + 1])), ns.add(fn(a[i], b[j + 1]))])

    grid(xs, zs, lambda x, z: (x, B / 2, z))
    grid(xs, yb, lambda x, y: (x, y, -D))
    grid(ye, zs, lambda y, z: (-L / 2, y, z))
    grid(ye, zs, lambda y, z: (L / 2, y, z))
    nodes = np.array(ns.xyz)
    panels = np.array(quads, dtype=np.int32)
    cen = np.tile([0.0, 0.0, -D / 2], (len(panels), 1))
    mesh = Mesh(nodes, _orient(nodes, panels, cen), isym=1)
    return Case(mesh, np.linspace(0.05, 2.5, n_omega), np.array([0.0, 45.0, 90.0]),
                six_dofs(), six_dofs(), rho=1025.0, g=9.81, depth=50.0, name="barge2400")


ICO_JITTER = 0.03   # tangential node jitter: panel areas within +-10% of the unjittered mesh


def config_two_spheres(n_omega=30, seed=3) -> Case:
    """Two floating spheres R=4 m, centres (+-10, 0, 0), 8,000 panels total.

    Each hull is a geodesic icosphere (frequency 12) cut at 0.055 radii below
    the centre (draft 3.78 m) and levelled onto the waterline, quadrangulated
    (three quads per triangle, 3,996 quads, the four largest halved: 4,000),
    with node jitter from `seed` that changes panel areas by up to 10%.
    """
    rng = np.random.default_rng(seed)
    a = icosphere_hull(4.0, 12, -0.055, (-10.0, 0.0), n_target=4000, jitter=ICO_JITTER, rng=rng)
    b = icosphere_hull(4.0, 12, -0.055, (10.0, 0.0), n_target=4000, jitter=ICO_JITTER, rng=rng)
    mesh = merge_meshes([a, b])
    dofs = six_dofs((-10.0, 0.0, 0.0), 1) + six_dofs((10.0, 0.0, 0.0), 2)
    return Case(mesh, np.linspace(0.2, 3.0, n_omega), np.array([0.0, 90.0]),
                dofs, list(dofs), rho=1025.0, g=9.81, depth=0.0, name="two_spheres8000")


def random_body(rng, n_min=200, n_max=3000):
    """One body of the batched/serving workloads: cylinder, box or sphere.

    Returns (mesh, depth) with dimensions U(2,30) m, draft U(1,15) m and a
    panel count drawn log-uniform in [n_min, n_max] (met approximately).
    """
    kind = int(rng.integers(0, 3))
    target = int(round(math.exp(rng.uniform(math.log(n_min), math.log(n_max)))))
    dim = float(rng.uniform(2.0, 30.0))
    draft = float(rng.uniform(1.0, 15.0))
    depth = 0.0 if rng.uniform() < 0.5 else float(rng.uniform(20.0, 200.0))
    if kind == 0:
        r = dim / 2
        # side n_t*n_z + bottom n_r*n_s with n_s = n_t/2
        area_side = 2 * math.pi * r * draft
        area_bot = math.pi * r * r
        h = math.sqrt((area_side + area_bot) / target)
        nt = max(8, 2 * int(round(math.pi * r / h)))
        nz = max(2, int(round(draft / h)))
        nr = max(1, int(round(r / h)))
        while nt * nz + nr * (nt // 2) > n_max and nt > 8:
            nt -= 2
        mesh = cylinder_mesh(r, draft, nt, nz, nr, max(4, nt // 2))
    elif kind == 1:
        length, beam = dim, float(rng.uniform(2.0, 30.0))
        area = 2 * (length + beam) * draft + length * beam
        h = math.sqrt(area / target)
        nx = max(2, int(round(length / h)))
        ny = max(2, int(round(beam / h)))
        nz = max(2, int(round(draft / h)))
        mesh = box_mesh(length, beam, draft, nx, ny, nz)
    else:
        r = dim / 2
        draft = min(draft, r)
        nlat = max(4, int(round(math.sqrt(target / 2.5))))
        nlon = max(8, int(round(target / nlat)))
        mesh = hemisphere_mesh(r, nlat, nlon, draft=draft)
    if depth > 0.0:
        depth = max(depth, 1.5 * draft + 5.0)
    return mesh, depth


def config_batch(n_bodies=256, n_omega=20, seed=4, n_min=200, n_max=3000):
    """Uneven-size batch: `n_bodies` random bodies, `n_omega` frequencies each."""
    rng = np.random.default_rng(seed)
    cases = []
    for b in range(n_bodies):
        mesh, depth = random_body(rng, n_min, n_max)
        cases.append(Case(mesh, np.linspace(0.1, 2.5, n_omega), np.array([0.0]),
                          six_dofs(), six_dofs(), depth=depth, name="body%03d" % b))
    return cases


def serving_stream(n_requests=10000, rate=100.0, seed=5, n_bodies=32, n_min=200, n_max=3000):
    """Poisson arrivals of (body index, omega, heading) solve requests.

    Returns (bodies [(mesh, depth)], arrivals_s, body_idx, omega, beta_deg).
    """
    rng = np.random.default_rng(seed)
    bodies = [random_body(rng, n_min, n_max) for _ in range(n_bodies)]
    gaps = rng.exponential(1.0 / rate, n_requests)
    t = np.cumsum(gaps)
    idx = rng.integers(0, n_bodies, n_requests)
    om = rng.uniform(0.1, 2.5, n_requests)
    beta = rng.uniform(0.0, 180.0, n_requests)
    return bodies, t, idx, om, beta
