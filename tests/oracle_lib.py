"""ctypes access to the CPU oracle (test infrastructure, oracle/nemoh_oracle.cpp).

Only the tests, the smoke check and bench.py's CPU-baseline leg use this.
"""
import ctypes
import os
import subprocess
import threading

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(ROOT, "oracle")
LIB_PATH = os.path.join(ORACLE_DIR, "_build", "libnemoh_oracle.so")
_lock = threading.Lock()
_lib = None

_d = ctypes.POINTER(ctypes.c_double)
_i = ctypes.POINTER(ctypes.c_int)


def build():
    src = os.path.join(ORACLE_DIR, "nemoh_oracle.cpp")
    if not os.path.exists(LIB_PATH) or os.path.getmtime(LIB_PATH) < os.path.getmtime(src):
        subprocess.run(["make", "-s", "-C", ORACLE_DIR], check=True)


def lib():
    global _lib
    with _lock:
        if _lib is None:
            build()
            L = ctypes.CDLL(LIB_PATH)
            L.nemoh_oracle_last_error.restype = ctypes.c_char_p
            L.nemoh_oracle_create.argtypes = [ctypes.POINTER(ctypes.c_void_p), ctypes.c_int, ctypes.c_int,
                                              ctypes.c_int, _d, _i, ctypes.c_double, ctypes.c_double,
                                              ctypes.c_double]
            L.nemoh_oracle_destroy.argtypes = [ctypes.c_void_p]
            L.nemoh_oracle_set_cache_s.argtypes = [ctypes.c_void_p, ctypes.c_int]
            L.nemoh_oracle_geometry.argtypes = [ctypes.c_void_p, _d, _d]
            L.nemoh_oracle_tables.argtypes = [ctypes.c_void_p, _d, _d, _d]
            L.nemoh_oracle_assemble.argtypes = [ctypes.c_void_p, ctypes.c_double, _d, _d, _d, _d, _i, _i]
            L.nemoh_oracle_solve_problem.argtypes = [ctypes.c_void_p, ctypes.c_double, _d, _d, _d, _d, _d, _d,
                                                     _i, _i]
            L.nemoh_oracle_get_nq.argtypes = [ctypes.c_void_p]
            L.nemoh_oracle_set_nq.argtypes = [ctypes.c_void_p, ctypes.c_int]
            L.nemoh_oracle_run_case.argtypes = [ctypes.c_char_p, ctypes.c_int, _d]
            L.nemoh_oracle_gg.argtypes = [ctypes.c_double] * 4 + [_d]
            L.nemoh_oracle_x0.argtypes = [ctypes.c_double]
            L.nemoh_oracle_x0.restype = ctypes.c_double
            L.nemoh_oracle_lisc.argtypes = [ctypes.c_double, ctypes.c_double, _i, _d, _d]
            L.nemoh_oracle_cint.argtypes = [ctypes.c_double, _d, _d]
            L.nemoh_oracle_gaussz_inverse.argtypes = [ctypes.c_int, _d, _d]
            L.nemoh_oracle_kochin.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                              ctypes.c_int, _d, ctypes.c_int, _d, _d, _d]
            L.nemoh_oracle_free_surface.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_int, _d,
                                                    ctypes.c_int, _d, _d, _d]
            _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(_d)


class OracleError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("oracle status %d: %s" % (code, msg))
        self.code = code


def _check(st):
    if st != 0:
        raise OracleError(st, lib().nemoh_oracle_last_error().decode())


class Oracle:
    """One Solver state (the reference's COM_VAR) on one mesh."""

    def __init__(self, nodes, panels, isym, rho, g, depth, cache_s=True):
        L = lib()
        self.nodes = np.ascontiguousarray(nodes, dtype=np.float64)
        self.panels = np.ascontiguousarray(panels, dtype=np.int32)
        self.n = len(self.panels)
        self.isym = isym
        h = ctypes.c_void_p()
        _check(L.nemoh_oracle_create(ctypes.byref(h), len(self.nodes), self.n, isym, _p(self.nodes),
                                     self.panels.ctypes.data_as(_i), rho, g, depth))
        self.h = h
        L.nemoh_oracle_set_cache_s(h, 1 if cache_s else 0)

    def __del__(self):
        if getattr(self, "h", None):
            lib().nemoh_oracle_destroy(self.h)
            self.h = None

    def geometry(self):
        out = np.zeros(8 * self.n)
        zer = ctypes.c_double()
        lib().nemoh_oracle_geometry(self.h, _p(out), ctypes.byref(zer))
        return out.reshape(8, self.n), zer.value

    def tables(self):
        xr, xz, apd = np.zeros(328), np.zeros(46), np.zeros(4 * 328 * 46)
        lib().nemoh_oracle_tables(self.h, _p(xr), _p(xz), _p(apd))
        return xr, xz, apd.reshape(4, 46, 328).transpose(0, 2, 1)

    def assemble(self, omega):
        n = self.n
        mats = [np.zeros((n, n), dtype=np.complex128, order="F") for _ in range(4)]
        mode, nexp = ctypes.c_int(), ctypes.c_int()
        _check(lib().nemoh_oracle_assemble(self.h, omega, *[m.ctypes.data_as(_d) for m in mats],
                                           ctypes.byref(mode), ctypes.byref(nexp)))
        return mats, mode.value, nexp.value

    def solve_problem(self, period, nvel):
        n = self.n
        nvel = np.ascontiguousarray(nvel, dtype=np.complex128)
        zigb, zigs, zpb, zps = (np.zeros(n, dtype=np.complex128) for _ in range(4))
        pres = np.zeros(n * 2 ** self.isym, dtype=np.complex128)
        nexp, fd = ctypes.c_int(), ctypes.c_int()
        _check(lib().nemoh_oracle_solve_problem(self.h, period, nvel.ctypes.data_as(_d),
                                                *[a.ctypes.data_as(_d) for a in (zigb, zigs, zpb, zps, pres)],
                                                ctypes.byref(nexp), ctypes.byref(fd)))
        return dict(zigb=zigb, zigs=zigs, zpb=zpb, zps=zps, pressure=pres, nexp=nexp.value, fd=fd.value)

    def kochin(self, period, theta, zigb, zigs=None, xeff=0.0, yeff=0.0):
        """COMPUTE_KOCHIN for given source strengths (n,) or (n, nprob): (ntheta, nprob)."""
        theta = np.ascontiguousarray(theta, dtype=np.float64)
        zigb = np.asfortranarray(np.asarray(zigb, dtype=np.complex128).reshape(self.n, -1))
        zigs = (np.asfortranarray(np.asarray(zigs, dtype=np.complex128).reshape(self.n, -1))
                if zigs is not None else np.zeros_like(zigb))
        out = np.zeros((len(theta), zigb.shape[1]), dtype=np.complex128, order="F")
        _check(lib().nemoh_oracle_kochin(self.h, period, xeff, yeff, len(theta), theta.ctypes.data_as(_d),
                                         zigb.shape[1], zigb.ctypes.data_as(_d), zigs.ctypes.data_as(_d),
                                         out.ctypes.data_as(_d)))
        return out

    def free_surface(self, period, xy, zigb, zigs=None):
        """ETA at the points (x, y, 0) of xy (npts, 2) for source strengths (n,)
        or (n, nprob): (npts, nprob) complex."""
        xy = np.ascontiguousarray(np.asarray(xy, dtype=np.float64).reshape(-1, 2))
        zigb = np.asfortranarray(np.asarray(zigb, dtype=np.complex128).reshape(self.n, -1))
        zigs = (np.asfortranarray(np.asarray(zigs, dtype=np.complex128).reshape(self.n, -1))
                if zigs is not None else np.zeros_like(zigb))
        out = np.zeros((xy.shape[0], zigb.shape[1]), dtype=np.complex128, order="F")
        _check(lib().nemoh_oracle_free_surface(self.h, period, xy.shape[0], xy.ctypes.data_as(_d), zigb.shape[1],
                                               zigb.ctypes.data_as(_d), zigs.ctypes.data_as(_d),
                                               out.ctypes.data_as(_d)))
        return out

    @property
    def nq(self):
        return lib().nemoh_oracle_get_nq(self.h)


def run_case(root, cache_s=True):
    secs = ctypes.c_double()
    _check(lib().nemoh_oracle_run_case(root.encode(), 1 if cache_s else 0, ctypes.byref(secs)))
    return secs.value


def gg(z, cex):
    out = np.zeros(2)
    lib().nemoh_oracle_gg(z.real, z.imag, cex.real, cex.imag, _p(out))
    return complex(out[0], out[1])


def x0(ak):
    return lib().nemoh_oracle_x0(ak)


def lisc(akh, amh):
    nexp = ctypes.c_int()
    a, r = np.zeros(31), np.zeros(31)
    _check(lib().nemoh_oracle_lisc(akh, amh, ctypes.byref(nexp), _p(a), _p(r)))
    return nexp.value, a, r


def cint(akk):
    q, c = np.zeros(101), np.zeros(101)
    n = lib().nemoh_oracle_cint(akk, _p(q), _p(c))
    return q[:n], c[:n]


def gaussz_inverse(a):
    a = np.asfortranarray(a, dtype=np.complex128)
    out = np.zeros_like(a, order="F")
    _check(lib().nemoh_oracle_gaussz_inverse(a.shape[0], a.ctypes.data_as(_d), out.ctypes.data_as(_d)))
    return out


def postproc(root):
    """The post-processor (postProcessor/Main.f90) on the case named by root/ID.dat."""
    L = lib()
    L.nemoh_oracle_postproc.argtypes = [ctypes.c_char_p]
    _check(L.nemoh_oracle_postproc(root.encode()))


def irf(w, damping, added_mass, ntime, dt):
    """Compute_IRF: damping/added mass (nw, nrad, nint) -> K (ntime, nrad, nint), A_inf (nrad, nint)."""
    L = lib()
    L.nemoh_oracle_irf.argtypes = [ctypes.c_int, _d, ctypes.c_int, ctypes.c_int, _d, _d, ctypes.c_int,
                                   ctypes.c_double, _d, _d]
    w = np.ascontiguousarray(w, dtype=np.float64)
    B = np.asfortranarray(damping, dtype=np.float64)
    A = np.asfortranarray(added_mass, dtype=np.float64)
    nw, nrad, nint = B.shape
    K = np.zeros((ntime, nrad, nint), order="F")
    ainf = np.zeros((nrad, nint), order="F")
    _check(L.nemoh_oracle_irf(nw, w.ctypes.data_as(_d), nrad, nint, B.ctypes.data_as(_d), A.ctypes.data_as(_d),
                              ntime, dt, K.ctypes.data_as(_d), ainf.ctypes.data_as(_d)))
    return K, ainf
