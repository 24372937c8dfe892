"""nemoh_b200: Nemoh's per-frequency BEM solve on an NVIDIA B200 (sm_100a).

Python access to the C-ABI of libnemoh_b200.so (include/nemoh_b200.h). The
interface mirrors the reference Solver's routines:

    Solver.set_mesh(...)            INITIALIZE + PRE_PROC_MESH
                                    (Solver/Core/INITIALIZATION.f90:28-69)
    Solver.solve_potential(T, nvel) SOLVE_POTENTIAL_INFD_DIRECT / _FD_DIRECT
                                    (SOLVE_BEM_INFD_DIRECT.f90:34, SOLVE_BEM_FD_DIRECT.f90:33)
                                    -> ZIGB, ZIGS, ZPB, ZPS, NEXP
    Solver.solve_bvp(T, nvel)       SOLVE_BVP pressure (SOLVE_BEM.f90:28-96)
    Solver.solve_frequencies(...)   all problems of many frequencies at once, with
                                    the force integration of Solver/NEMOH.f90:137-141

There is no CPU fallback: without the built library or a CUDA device every
call raises.
"""
import ctypes
import os

import numpy as np

__all__ = ["Solver", "NemohError", "FP64", "MIXED", "load_library", "library_path"]

FP64 = 0
MIXED = 1

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libnemoh_b200.so")
_lib = None

_d = ctypes.POINTER(ctypes.c_double)
_i = ctypes.POINTER(ctypes.c_int)
_vp = ctypes.c_void_p

_ERRNAMES = {1: "EINVAL", 2: "EPANEL_AREA", 3: "EPIVOT", 4: "EOMEGA", 5: "ELISC", 6: "ESPRBM",
             7: "EDISPERSION", 8: "EAKZ", 9: "EIO", 10: "EHOUSRS", 20: "ECUDA", 21: "ENOMEM",
             22: "ENODEV", 23: "ECAPACITY", 30: "ETIMEOUT"}


class NemohError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("nemoh_b200 %s (%d): %s" % (_ERRNAMES.get(code, "?"), code, msg))
        self.code = code


def library_path():
    return _LIB_PATH


def load_library():
    """Load libnemoh_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(_LIB_PATH):
        raise RuntimeError("libnemoh_b200.so is not built (run python -m nemoh_b200.build)")
    L = ctypes.CDLL(_LIB_PATH)
    L.nemoh_b200_last_error.restype = ctypes.c_char_p
    L.nemoh_b200_last_error.argtypes = [_vp]
    L.nemoh_b200_create.argtypes = [ctypes.POINTER(_vp), ctypes.c_int, ctypes.c_int]
    L.nemoh_b200_destroy.argtypes = [_vp]
    L.nemoh_b200_set_mesh.argtypes = [_vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, _d, _i,
                                      ctypes.c_double, ctypes.c_double, ctypes.c_double]
    L.nemoh_b200_solve_problem.argtypes = [_vp, ctypes.c_double, _d, _d, _d, _d, _d, _i]
    L.nemoh_b200_solve_frequencies.argtypes = [_vp, ctypes.c_int, _d, ctypes.c_int, _d, ctypes.c_int, _d, _d]
    L.nemoh_b200_solve_frequencies_device.argtypes = [_vp, ctypes.c_int, _d, ctypes.c_int, _vp, ctypes.c_int,
                                                      _vp, _vp, _vp]
    L.nemoh_b200_assemble.argtypes = [_vp, ctypes.c_double, _d, _d, _d, _d, _i]
    L.nemoh_b200_get_tables.argtypes = [_vp, _d, _d, _d]
    L.nemoh_b200_get_geometry.argtypes = [_vp, _d, _d]
    L.nemoh_b200_last_timings.argtypes = [_vp, _d, _d, _d]
    L.nemoh_b200_last_factor_ms.argtypes = [_vp, _d]
    L.nemoh_b200_fallback_count.argtypes = [_vp, ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(ctypes.c_longlong)]
    L.nemoh_b200_last_refinement.argtypes = [_vp, _i, _d]
    L.nemoh_b200_launch_count.argtypes = [_vp]
    L.nemoh_b200_body_conditions.argtypes = [_vp, _i, ctypes.c_double, ctypes.c_double, ctypes.c_int, _d, ctypes.c_int,
                                             _d, ctypes.c_int, _i, _i, _d, _d, ctypes.c_int, _i, _i, _d, _d, _d, _d,
                                             _d]
    L.nemoh_b200_body_conditions_device.argtypes = [_vp, _i, ctypes.c_double, ctypes.c_double, ctypes.c_int, _d,
                                                    ctypes.c_int, _d, ctypes.c_int, _i, _i, _d, _d, ctypes.c_int, _i,
                                                    _i, _d, _d, _vp, _vp, _vp, _vp]
    L.nemoh_b200_kochin.argtypes = [_vp, ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_int, _d,
                                    ctypes.c_int, _d, _d, _d]
    L.nemoh_b200_free_surface.argtypes = [_vp, ctypes.c_double, ctypes.c_int, _d, ctypes.c_int, _d, _d, _d]
    L.nemoh_b200_irf.argtypes = [_vp, ctypes.c_int, _d, ctypes.c_int, ctypes.c_int, _d, _d, ctypes.c_int,
                                 ctypes.c_double, _d, _d]
    L.nemoh_b200_launch_count.restype = ctypes.c_longlong
    L.nemoh_b200_add_body.argtypes = [_vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, _d, _i, ctypes.c_double,
                                      ctypes.c_double, ctypes.c_double, ctypes.c_int, _d, _i]
    L.nemoh_b200_body_count.argtypes = [_vp]
    L.nemoh_b200_prepare_bodies.argtypes = [_vp]
    L.nemoh_b200_set_autotune.argtypes = [ctypes.c_int]
    L.nemoh_b200_solve_bodies.argtypes = [_vp, ctypes.c_int, _i, _d, ctypes.c_int, _d, _d]
    L.nemoh_b200_solve_bodies_device.argtypes = [_vp, ctypes.c_int, _i, _d, ctypes.c_int, _vp, _vp, _vp]
    L.nemoh_b200_set_body_dofs.argtypes = [_vp, ctypes.c_int, ctypes.c_int, _i, _d, _d]
    L.nemoh_b200_set_graphs.argtypes = [_vp, ctypes.c_int]
    L.nemoh_b200_graph_stats.argtypes = [_vp, ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(ctypes.c_longlong)]
    L.nemoh_b200_solve_requests.argtypes = [_vp, ctypes.c_int, _i, _d, _d, _d]
    L.nemoh_b200_diag_dispersion_root.argtypes = [ctypes.c_double, _d]
    L.nemoh_b200_diag_exponential_fit.argtypes = [ctypes.c_double, ctypes.c_double, _i, _d, _d]
    L.nemoh_b200_diag_theta_quadrature.argtypes = [ctypes.c_double, _d, _d]
    L.nemoh_b200_diag_stencil_thresholds.argtypes = [_d, _d, _d]
    _lib = L
    return L


def _p(a):
    return a.ctypes.data_as(_d)


def _cplx(a, n=None):
    a = np.ascontiguousarray(a, dtype=np.complex128)
    if n is not None and a.size != n:
        raise ValueError("expected %d complex values, got %d" % (n, a.size))
    return a


class Solver:
    """One solver context on one GPU (the reference's COM_VAR state)."""

    def __init__(self, device=0, precision=FP64):
        L = load_library()
        h = _vp()
        st = L.nemoh_b200_create(ctypes.byref(h), int(device), int(precision))
        if st:
            raise NemohError(st, "nemoh_b200_create failed (no CUDA device?)")
        self._h = h
        self.precision = precision
        self.nfa = 0
        self.isym = 0

    def close(self):
        if getattr(self, "_h", None):
            load_library().nemoh_b200_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _check(self, st):
        if st:
            raise NemohError(st, load_library().nemoh_b200_last_error(self._h).decode())

    @property
    def launches(self):
        return int(load_library().nemoh_b200_launch_count(self._h))

    # -- INITIALIZE -----------------------------------------------------------
    def set_mesh(self, nodes, panels, isym, rho, g, depth):
        nodes = np.ascontiguousarray(nodes, dtype=np.float64)
        panels = np.ascontiguousarray(panels, dtype=np.int32)
        self._check(load_library().nemoh_b200_set_mesh(self._h, len(nodes), len(panels), int(isym), _p(nodes),
                                                       panels.ctypes.data_as(_i), rho, g, depth))
        self.nfa = len(panels)
        self.isym = 1 if isym == 1 else 0
        self.rho = rho

    def set_case(self, case):
        """Mesh and environment of a nemoh_b200.cases.Case or CaseArrays."""
        mesh = getattr(case, "mesh", None)
        if mesh is not None:
            self.set_mesh(mesh.nodes, mesh.panels, mesh.isym, case.rho, case.g, case.depth)
        else:
            self.set_mesh(case.nodes, case.panels, case.isym, case.rho, case.g, case.depth)

    # -- SOLVE_POTENTIAL_*_DIRECT ---------------------------------------------
    def solve_potential(self, period, nvel):
        n = self.nfa
        nvel = _cplx(nvel, n * 2 ** self.isym)
        out = [np.zeros(n, dtype=np.complex128) for _ in range(4)]
        nexp = ctypes.c_int()
        self._check(load_library().nemoh_b200_solve_problem(self._h, float(period), _p(nvel),
                                                            *[_p(a) for a in out], ctypes.byref(nexp)))
        zigb, zigs, zpb, zps = out
        return dict(zigb=zigb, zigs=zigs, zpb=zpb, zps=zps, nexp=nexp.value)

    def solve_bvp(self, period, nvel):
        """PRESSURE = RHO*i*W*[ZPB; ZPS] (SOLVE_BEM.f90:91-96)."""
        r = self.solve_potential(period, nvel)
        w = 2.0 * np.pi / period
        p = self.rho * 1j * w * r["zpb"]
        if self.isym:
            p = np.concatenate([p, self.rho * 1j * w * r["zps"]])
        return p

    # -- batched frequencies ----------------------------------------------------
    def solve_frequencies(self, omegas, nvel, nds):
        """nvel: (2^s N, nrhs, nomega) complex; nds: (nint, 2^s N). Returns force (nint, nrhs, nomega)."""
        omegas = np.ascontiguousarray(omegas, dtype=np.float64)
        nvel = np.asfortranarray(nvel, dtype=np.complex128)
        nds = np.asfortranarray(nds, dtype=np.float64)
        nc, nrhs, nw = nvel.shape
        nint = nds.shape[0]
        if nc != self.nfa * 2 ** self.isym or nw != len(omegas) or nds.shape[1] != nc:
            raise ValueError("shape mismatch")
        force = np.zeros((nint, nrhs, nw), dtype=np.complex128, order="F")
        self._check(load_library().nemoh_b200_solve_frequencies(self._h, nw, _p(omegas), nrhs,
                                                                nvel.ctypes.data_as(_d), nint,
                                                                nds.ctypes.data_as(_d), force.ctypes.data_as(_d)))
        return force

    def solve_frequencies_device(self, omegas, nvel_ptr, nrhs, nint, nds_ptr, force_ptr, stream=0):
        omegas = np.ascontiguousarray(omegas, dtype=np.float64)
        self._check(load_library().nemoh_b200_solve_frequencies_device(
            self._h, len(omegas), _p(omegas), int(nrhs), _vp(nvel_ptr), int(nint), _vp(nds_ptr),
            _vp(force_ptr), _vp(stream)))

    # -- resident bodies and cross-body batches ------------------------------
    def add_body(self, case, nds=None):
        """Keep a body (mesh and environment of a cases.Case, generalised
        normals nds (nint, 2^s N), by default those of the case) resident on
        the device; returns its id."""
        from . import cases as C
        m = case.mesh
        nodes = np.ascontiguousarray(m.nodes, dtype=np.float64)
        panels = np.ascontiguousarray(m.panels, dtype=np.int32)
        if nds is None:
            nds = C.generalised_normals(case)
        nds = np.asfortranarray(nds, dtype=np.float64)
        bid = ctypes.c_int()
        self._check(load_library().nemoh_b200_add_body(self._h, len(nodes), len(panels), int(m.isym), _p(nodes),
                                                       panels.ctypes.data_as(_i), case.rho, case.g, case.depth,
                                                       nds.shape[0], _p(nds), ctypes.byref(bid)))
        if not hasattr(self, "_bodies"):
            self._bodies = []
        self._bodies.append((len(panels) * (2 if m.isym == 1 else 1), nds.shape[0]))
        return bid.value

    def solve_bodies(self, bodies, omegas, nvels):
        """(body, omega) items with their right-hand sides nvels[i] ((2^s N_i, nrhs)
        complex, the same nrhs for all); returns the forces, one (nint_i, nrhs)
        array per item."""
        bodies = np.ascontiguousarray(bodies, dtype=np.int32)
        omegas = np.ascontiguousarray(omegas, dtype=np.float64)
        nrhs = nvels[0].shape[1]
        for b, v in zip(bodies, nvels):
            if not 0 <= b < len(getattr(self, "_bodies", ())):
                raise NemohError(1, "unknown body %d" % b)
            if v.shape != (self._bodies[b][0], nrhs):
                raise ValueError("right-hand sides of body %d: expected %s, got %s" % (b, (self._bodies[b][0], nrhs),
                                                                                    v.shape))
        flat = np.concatenate([np.asfortranarray(v, dtype=np.complex128).ravel(order="F") for v in nvels])
        sizes = [self._bodies[b][1] * nrhs for b in bodies]
        force = np.zeros(sum(sizes), dtype=np.complex128)
        self._check(load_library().nemoh_b200_solve_bodies(self._h, len(bodies), bodies.ctypes.data_as(_i),
                                                           _p(omegas), nrhs, _p(flat), _p(force)))
        out, o = [], 0
        for b, sz in zip(bodies, sizes):
            out.append(force[o:o + sz].reshape((self._bodies[b][1], nrhs), order="F"))
            o += sz
        return out

    def set_graphs(self, on=True):
        """Capture repeated cross-body batches into CUDA graphs and replay them."""
        self._check(load_library().nemoh_b200_set_graphs(self._h, 1 if on else 0))

    def graph_stats(self):
        cap, rep = ctypes.c_longlong(), ctypes.c_longlong()
        load_library().nemoh_b200_graph_stats(self._h, ctypes.byref(cap), ctypes.byref(rep))
        return cap.value, rep.value

    def set_body_dofs(self, body, dofs):
        """Radiation DOFs (cases.Dof list) of a resident body's serving requests."""
        kind = np.array([d.icase for d in dofs], dtype=np.int32)
        direc = np.ascontiguousarray([d.direction for d in dofs], dtype=np.float64).reshape(-1)
        axis = np.ascontiguousarray([d.axis for d in dofs], dtype=np.float64).reshape(-1)
        self._check(load_library().nemoh_b200_set_body_dofs(self._h, int(body), len(dofs), kind.ctypes.data_as(_i),
                                                            _p(direc), _p(axis)))
        self._bodies[body] = self._bodies[body][:2] + (len(dofs),)

    def solve_requests(self, bodies, omegas, betas_rad):
        """Serving requests (body, omega, heading): right-hand sides built on
        the device; returns per request the forces (nint, 1 + ndof): the
        diffraction problem, then the radiation DOFs."""
        bodies = np.ascontiguousarray(bodies, dtype=np.int32)
        omegas = np.ascontiguousarray(omegas, dtype=np.float64)
        betas = np.ascontiguousarray(betas_rad, dtype=np.float64)
        nrhs = 1 + self._bodies[bodies[0]][2]
        sizes = [self._bodies[b][1] * nrhs for b in bodies]
        force = np.zeros(sum(sizes), dtype=np.complex128)
        self._check(load_library().nemoh_b200_solve_requests(self._h, len(bodies), bodies.ctypes.data_as(_i),
                                                             _p(omegas), _p(betas), _p(force)))
        out, o = [], 0
        for b, sz in zip(bodies, sizes):
            out.append(force[o:o + sz].reshape((self._bodies[b][1], nrhs), order="F"))
            o += sz
        return out

    def solve_bodies_device(self, bodies, omegas, nrhs, nvel_ptr, force_ptr, stream=0):
        bodies = np.ascontiguousarray(bodies, dtype=np.int32)
        omegas = np.ascontiguousarray(omegas, dtype=np.float64)
        self._check(load_library().nemoh_b200_solve_bodies_device(
            self._h, len(bodies), bodies.ctypes.data_as(_i), _p(omegas), int(nrhs), _vp(nvel_ptr), _vp(force_ptr),
            _vp(stream)))

    def last_timings(self):
        a, f, s, lu = ctypes.c_double(), ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        L = load_library()
        L.nemoh_b200_last_timings(self._h, ctypes.byref(a), ctypes.byref(f), ctypes.byref(s))
        L.nemoh_b200_last_factor_ms(self._h, ctypes.byref(lu))
        return dict(assemble_ms=a.value, factor_ms=f.value, solve_ms=s.value, lu_ms=lu.value)

    def prepare_bodies(self):
        """Evaluate the resident bodies' Rankine parts now (each depth regime
        they can meet), so that no later solve pays for them."""
        self._check(load_library().nemoh_b200_prepare_bodies(self._h))

    def fallback_count(self):
        """(batches that fell back to FP64 factors, systems re-solved in partial fallbacks)"""
        nb_, ns = ctypes.c_longlong(), ctypes.c_longlong()
        load_library().nemoh_b200_fallback_count(self._h, ctypes.byref(nb_), ctypes.byref(ns))
        return nb_.value, ns.value

    def last_refinement(self):
        it, res = ctypes.c_int(), ctypes.c_double()
        load_library().nemoh_b200_last_refinement(self._h, ctypes.byref(it), ctypes.byref(res))
        return it.value, res.value

    # -- pre-processor on the device ------------------------------------------
    def body_conditions(self, case):
        """NVEL (2^s N, Nproblems) in the pre-processor's problem order, NDS
        (Nint, 2^s N) and Froude-Krylov forces (Nw, Nbeta, Nint), computed on the
        GPU for `case` (its mesh must be the current one)."""
        nc = self.nfa * 2 ** self.isym
        nw, nb, nr, nf = len(case.omegas), len(case.betas_deg), len(case.rad), len(case.force)
        nvel = np.zeros((nc, nb + nr, nw), dtype=np.complex128, order="F")
        nds = np.zeros((nf, nc), dtype=np.float64, order="F")
        fk = np.zeros((nf, nb, nw), dtype=np.complex128, order="F")
        args, _keep = self._body_condition_args(case)
        self._check(load_library().nemoh_b200_body_conditions(
            self._h, *args, nvel.ctypes.data_as(_d), nds.ctypes.data_as(_d), fk.ctypes.data_as(_d)))
        return nvel.reshape(nc, (nb + nr) * nw, order="F"), nds, fk.transpose(2, 1, 0)

    def body_conditions_device(self, case, nvel_ptr, nds_ptr, fk_ptr, stream=0):
        """The same outputs written to device memory of the context's device,
        column-major: nvel (2^s N, Nbeta + Nrad, Nw) complex, nds (Nint, 2^s N)
        real, fk (Nint, Nbeta, Nw) complex; ordered after the work on `stream`."""
        args, _keep = self._body_condition_args(case)
        self._check(load_library().nemoh_b200_body_conditions_device(
            self._h, *args, _vp(nvel_ptr), _vp(nds_ptr), _vp(fk_ptr), _vp(stream)))

    @staticmethod
    def _body_condition_args(case):
        """Leading C arguments of the body-conditions entry points (and the
        arrays they point into, which must outlive the call)."""
        def spec(dofs):
            kind = np.array([d.icase for d in dofs] or [1], dtype=np.int32)
            body = np.array([d.body for d in dofs] or [1], dtype=np.int32)
            dr = np.array([d.direction for d in dofs] or [(0, 0, 0)], dtype=np.float64).ravel()
            ax = np.array([d.axis for d in dofs] or [(0, 0, 0)], dtype=np.float64).ravel()
            return kind, body, dr, ax
        nw, nb, nr, nf = len(case.omegas), len(case.betas_deg), len(case.rad), len(case.force)
        rk, rb, rd, ra = spec(case.rad)
        fk_, fb, fd, fa = spec(case.force)
        om = np.ascontiguousarray(case.omegas, dtype=np.float64)
        beta = np.ascontiguousarray(np.asarray(case.betas_deg, dtype=np.float64) * np.pi / 180.0)
        if not nb:
            beta = np.zeros(1)
        pb = np.ascontiguousarray(case.mesh.body, dtype=np.int32)
        ip = lambda a: a.ctypes.data_as(_i)
        args = (ip(pb), float(case.xeff), float(case.yeff), nw, _p(om), nb, _p(beta), nr, ip(rk), ip(rb), _p(rd),
                _p(ra), nf, ip(fk_), ip(fb), _p(fd), _p(fa))
        return args, (rk, rb, rd, ra, fk_, fb, fd, fa, om, beta, pb)

    # -- COMPUTE_KOCHIN ---------------------------------------------------------
    def kochin(self, period, theta, zigb, zigs=None, xeff=0.0, yeff=0.0):
        """Kochin function H(theta) of problems solved at `period` from their source
        strengths (nfa,) or (nfa, nprob); returns (ntheta, nprob) complex."""
        theta = np.ascontiguousarray(theta, dtype=np.float64)
        zigb = np.asfortranarray(np.asarray(zigb, dtype=np.complex128).reshape(self.nfa, -1))
        nprob = zigb.shape[1]
        zigs = (np.asfortranarray(np.asarray(zigs, dtype=np.complex128).reshape(self.nfa, -1))
                if zigs is not None else np.zeros_like(zigb))
        out = np.zeros((len(theta), nprob), dtype=np.complex128, order="F")
        self._check(load_library().nemoh_b200_kochin(self._h, float(period), float(xeff), float(yeff), len(theta),
                                                     _p(theta), nprob, zigb.ctypes.data_as(_d),
                                                     zigs.ctypes.data_as(_d), out.ctypes.data_as(_d)))
        return out

    # -- COMPUTE_POTENTIAL_DOMAIN on the free surface --------------------------
    def free_surface(self, period, xy, zigb, zigs=None):
        """Free-surface elevation ETA = i W/G PHI at the points (x, y, 0) of xy
        (npts, 2) for problems solved at `period` from their source strengths
        (nfa,) or (nfa, nprob); returns (npts, nprob) complex."""
        xy = np.ascontiguousarray(np.asarray(xy, dtype=np.float64).reshape(-1, 2))
        zigb = np.asfortranarray(np.asarray(zigb, dtype=np.complex128).reshape(self.nfa, -1))
        nprob = zigb.shape[1]
        zigs = (np.asfortranarray(np.asarray(zigs, dtype=np.complex128).reshape(self.nfa, -1))
                if zigs is not None else np.zeros_like(zigb))
        out = np.zeros((xy.shape[0], nprob), dtype=np.complex128, order="F")
        self._check(load_library().nemoh_b200_free_surface(self._h, float(period), xy.shape[0], _p(xy), nprob,
                                                           zigb.ctypes.data_as(_d), zigs.ctypes.data_as(_d),
                                                           out.ctypes.data_as(_d)))
        return out

    # -- post-processor: Compute_IRF -------------------------------------------
    def irf(self, w, damping, added_mass, ntime, dt):
        """Impulse response functions K (ntime, nrad, nint) at t = i dt and the
        infinite-frequency added mass (nrad, nint) from damping and added mass
        (nw, nrad, nint) at the frequencies w (postProcessor/IRF.f90:100-127)."""
        w = np.ascontiguousarray(w, dtype=np.float64)
        B = np.asfortranarray(damping, dtype=np.float64)
        A = np.asfortranarray(added_mass, dtype=np.float64)
        nw, nrad, nint = B.shape
        if A.shape != B.shape or len(w) != nw:
            raise ValueError("damping, added mass and w must agree in shape")
        K = np.zeros((int(ntime), nrad, nint), order="F")
        ainf = np.zeros((nrad, nint), order="F")
        self._check(load_library().nemoh_b200_irf(self._h, nw, _p(w), nrad, nint, B.ctypes.data_as(_d),
                                                  A.ctypes.data_as(_d), int(ntime), float(dt), K.ctypes.data_as(_d),
                                                  ainf.ctypes.data_as(_d)))
        return K, ainf

    # -- diagnostics -----------------------------------------------------------
    def assemble(self, omega):
        n = self.nfa
        mats = [np.zeros((n, n), dtype=np.complex128, order="F") for _ in range(4)]
        mode = ctypes.c_int()
        self._check(load_library().nemoh_b200_assemble(self._h, float(omega), *[m.ctypes.data_as(_d) for m in mats],
                                                       ctypes.byref(mode)))
        return mats, mode.value

    def tables(self):
        xr, xz, apd = np.zeros(328), np.zeros(46), np.zeros(4 * 328 * 46)
        self._check(load_library().nemoh_b200_get_tables(self._h, _p(xr), _p(xz), _p(apd)))
        return xr, xz, apd.reshape(4, 46, 328).transpose(0, 2, 1)

    def geometry(self):
        out = np.zeros(8 * self.nfa)
        zer = ctypes.c_double()
        self._check(load_library().nemoh_b200_get_geometry(self._h, _p(out), ctypes.byref(zer)))
        return out.reshape(8, self.nfa), zer.value


# host-side setup checks (no device needed)
def dispersion_root(ak):
    r = ctypes.c_double()
    st = load_library().nemoh_b200_diag_dispersion_root(float(ak), ctypes.byref(r))
    if st:
        raise NemohError(st, "dispersion root")
    return r.value


def exponential_fit(akh, amh):
    n = ctypes.c_int()
    a, r = np.zeros(31), np.zeros(31)
    st = load_library().nemoh_b200_diag_exponential_fit(float(akh), float(amh), ctypes.byref(n), _p(a), _p(r))
    if st:
        raise NemohError(st, "exponential fit")
    return n.value, a, r


def theta_quadrature(akk):
    q, c = np.zeros(101), np.zeros(101)
    n = load_library().nemoh_b200_diag_theta_quadrature(float(akk), _p(q), _p(c))
    return q[:n], c[:n]


def stencil_thresholds():
    a, b, c = np.zeros(48), np.zeros(48), np.zeros(48)
    load_library().nemoh_b200_diag_stencil_thresholds(_p(a), _p(b), _p(c))
    return a, b, c


def sweep_timeout_check(device=0):
    """Bounded-wait check of the dataflow triangular sweep: one launch whose
    only item waits on a ready flag that nothing raises. Returns the status
    word the kernel left (31: the wait ran out) and the launch's duration in
    ms; the device stays usable."""
    L = load_library()
    L.nemoh_b200_diag_sweep_timeout.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                                                ctypes.POINTER(ctypes.c_double)]
    st, ms = ctypes.c_int(), ctypes.c_double()
    rc = L.nemoh_b200_diag_sweep_timeout(int(device), ctypes.byref(st), ctypes.byref(ms))
    if rc:
        raise NemohError(rc, "sweep timeout check")
    return st.value, ms.value


def sweep_choice(n, nsys, nrhs, single):
    """The sweep the autotuner chose for a batch shape (0: not tuned yet;
    1, 2, 4, 8: cluster sweep with that cluster size; 16: dataflow sweep) and
    the number of shapes tuned so far in this process."""
    L = load_library()
    L.nemoh_b200_diag_sweep_tuning.argtypes = [ctypes.POINTER(ctypes.c_longlong), ctypes.c_int, ctypes.c_int,
                                               ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_int)]
    keys, cs = ctypes.c_longlong(), ctypes.c_int()
    L.nemoh_b200_diag_sweep_tuning(ctypes.byref(keys), int(n), int(nsys), int(nrhs), int(bool(single)),
                                   ctypes.byref(cs))
    return cs.value, keys.value


def set_autotune(on):
    """Autotuning of the triangular sweep, process-wide (on by default): off, a
    batch shape not tuned yet is solved with the default sweep."""
    load_library().nemoh_b200_set_autotune(int(bool(on)))
