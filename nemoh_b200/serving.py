"""Continuous-batching solve server on one GPU.

Requests are (body, omega, heading) solves of Nemoh's per-frequency BEM
problem: 6 radiation DOFs plus the diffraction problem at one heading, i.e.
one (mesh, omega) system with 7 right-hand sides, whose result is the force
matrix (nint x 7) of Solver/NEMOH.f90:137-141.

Design:
* workers -- each owns one library context (its own CUDA stream and device
  workspace), so batches of different workers overlap on the device;
* meshes stay resident: a worker keeps its current mesh and switches with
  `set_mesh` (panel geometry on the device, no table rebuild);
* admission by HBM footprint: a batch takes at most as many frequencies as
  fit the worker's share of device memory (two complex128 N x N matrices per
  symmetry class plus workspace per frequency);
* workspace reserved up front: each worker first solves the largest body at
  `reserve` frequencies, so that later batches of up to that many frequencies
  find their device buffers in place (growing a buffer frees the old one, and
  cudaFree waits for every stream on the device, stalling the other workers);
* continuous batching: whenever a worker is free it takes the body of the
  oldest waiting request and every request of that body that has arrived,
  up to its admission limit; requests that arrive while others run join the
  next batch as soon as a worker frees up.

Radiation right-hand sides do not depend on omega and are built once per
body; the diffraction right-hand side of each request is built on the host
(pre-processor formulas, cases.py).
"""
import collections
import dataclasses
import math
import threading
import time
from typing import List, Optional

import numpy as np

from . import FP64, MIXED, Solver  # noqa: F401
from . import cases as C


@dataclasses.dataclass
class Request:
    rid: int
    body: int
    omega: float
    beta_deg: float
    arrival: float = 0.0          # seconds from the start of the run
    start: float = 0.0
    done: float = 0.0
    force: Optional[np.ndarray] = None   # (nint, 7): 6 radiation DOFs, then diffraction
    error: Optional[str] = None          # set when the request's batch failed


class Body:
    """One resident body: mesh, environment, generalised normals, radiation RHS."""

    def __init__(self, mesh: C.Mesh, depth: float, rho=1025.0, g=9.81):
        self.case = C.Case(mesh, np.array([1.0]), np.array([0.0]), C.six_dofs(), C.six_dofs(), rho=rho, g=g,
                           depth=depth)
        self.mesh = mesh
        self.nds = np.asfortranarray(C.generalised_normals(self.case))
        xm, n, a = C.panel_quantities(mesh)
        self._xm, self._n = xm, n
        self.rad = np.stack([C._dof_vector(mesh, xm, n, a, d, False) for d in self.case.rad], axis=1)

    @property
    def npanels(self):
        return self.mesh.npanels

    def rhs(self, omega, beta_deg):
        """(2^s N, 7) right-hand sides: 6 radiation DOFs then the diffraction problem."""
        k = C.wavenumber(omega, self.case.g, self.case.depth)
        beta = beta_deg * math.pi / 180.0
        xm, n = self._xm, self._n
        _, vx, vy, vz = C._wave(self.case, k, omega, beta, xm[:, 0], xm[:, 1], xm[:, 2])
        diff = -(vx * n[:, 0] + vy * n[:, 1] + vz * n[:, 2])
        if self.mesh.isym == 1:
            _, vx, vy, vz = C._wave(self.case, k, omega, beta, xm[:, 0], -xm[:, 1], xm[:, 2])
            diff = np.concatenate([diff, -(vx * n[:, 0] - vy * n[:, 1] + vz * n[:, 2])])
        return np.concatenate([self.rad.astype(np.complex128), diff[:, None]], axis=1)

    def bytes_per_frequency(self):
        n = self.npanels
        cls = 2 if self.mesh.isym else 1
        return cls * n * n * 16 * 2 + cls * n * n * 8 + cls * n * 7 * 16 * 6


class ServeError(RuntimeError):
    """Raised by SolveServer.run when batches failed: `failed` holds their
    requests (each with its `error` text), `done` the requests that were served."""

    def __init__(self, failed, done):
        first = failed[0]
        super().__init__("%d of %d requests failed; first (request %d): %s" %
                         (len(failed), len(failed) + len(done), first.rid, first.error))
        self.failed = failed
        self.done = done


class SolveServer:
    """Serve a stream of requests on one GPU with `workers` concurrent contexts."""

    def __init__(self, bodies: List[Body], device=0, precision=MIXED, workers=2, memory_fraction=0.6,
                 solver_factory=None, memory_bytes=None, reserve=0):
        self.bodies = bodies
        self.device = device
        self.precision = precision
        self.nworkers = workers
        self.memory_fraction = memory_fraction
        self._lock = threading.Condition()
        self._pending = collections.deque()
        self._done: List[Request] = []
        self._failed: List[Request] = []
        self._feeding = False
        make = solver_factory or (lambda: Solver(device, precision))
        self._solvers = [make() for _ in range(workers)]
        self._current = [None] * workers
        self.batches = []   # (worker, body, nreq, t0, t1)
        free = memory_bytes
        if free is None:
            import torch
            free, _ = torch.cuda.mem_get_info(device)
        self._budget = free * memory_fraction / workers
        if reserve > 0 and bodies:
            big = max(range(len(bodies)), key=lambda b: bodies[b].bytes_per_frequency())
            body = bodies[big]
            k = min(reserve, self.admission(body))
            omegas = np.linspace(0.5, 2.0, k)
            nvel = np.stack([body.rhs(w, 0.0) for w in omegas], axis=2)
            for w, s in enumerate(self._solvers):
                s.set_case(body.case)
                s.solve_frequencies(omegas, nvel, body.nds)
                self._current[w] = big

    def close(self):
        for s in self._solvers:
            s.close()

    def admission(self, body: Body):
        """Frequencies per batch that fit this worker's share of HBM."""
        return max(1, int(self._budget // body.bytes_per_frequency()))

    def _take_batch(self, w):
        with self._lock:
            while not self._pending:
                if not self._feeding:
                    return None
                self._lock.wait(timeout=0.005)
            head = self._pending[0]
            b = head.body
            cap = self.admission(self.bodies[b])
            batch, keep = [], collections.deque()
            while self._pending:
                r = self._pending.popleft()
                if r.body == b and len(batch) < cap:
                    batch.append(r)
                else:
                    keep.append(r)
            self._pending = keep
            return batch

    def _worker(self, w, t0):
        s = self._solvers[w]
        while True:
            batch = self._take_batch(w)
            if batch is None:
                return
            b = batch[0].body
            body = self.bodies[b]
            tb = time.perf_counter() - t0
            for r in batch:
                r.start = tb
            try:
                if self._current[w] != b:
                    self._current[w] = None
                    s.set_case(body.case)
                    self._current[w] = b
                omegas = np.array([r.omega for r in batch])
                nvel = np.stack([body.rhs(r.omega, r.beta_deg) for r in batch], axis=2)
                force = s.solve_frequencies(omegas, nvel, body.nds)
            except Exception as e:   # the batch fails as a whole; the worker serves on
                td = time.perf_counter() - t0
                for r in batch:
                    r.error = "%s: %s" % (type(e).__name__, e)
                    r.done = td
                with self._lock:
                    self._failed.extend(batch)
                continue
            td = time.perf_counter() - t0
            for i, r in enumerate(batch):
                r.force = force[:, :, i]
                r.done = td
            with self._lock:
                self._done.extend(batch)
                self.batches.append((w, b, len(batch), tb, td))

    def run(self, requests: List[Request], realtime=True):
        """Feed requests at their arrival times (or all at once) and wait for all results."""
        self._done = []
        self._failed = []
        self.batches = []
        reqs = sorted(requests, key=lambda r: r.arrival)
        self._feeding = True
        t0 = time.perf_counter()
        threads = [threading.Thread(target=self._worker, args=(w, t0), daemon=True) for w in range(self.nworkers)]
        for t in threads:
            t.start()
        for r in reqs:
            if realtime:
                dt = r.arrival - (time.perf_counter() - t0)
                if dt > 0:
                    time.sleep(dt)
            with self._lock:
                self._pending.append(r)
                self._lock.notify_all()
        with self._lock:
            self._feeding = False
            self._lock.notify_all()
        for t in threads:
            t.join()
        wall = time.perf_counter() - t0
        if self._failed:
            raise ServeError(self._failed, self._done)
        if len(self._done) != len(reqs):
            raise RuntimeError("served %d of %d requests" % (len(self._done), len(reqs)))
        return self._done, wall


def latency_stats(done: List[Request], wall: float, expected: Optional[int] = None):
    """p50/p99/mean latency (arrival to result) and throughput; with `expected`
    the number of served requests must match it."""
    if expected is not None and len(done) != expected:
        raise RuntimeError("latency over %d requests, %d expected" % (len(done), expected))
    if any(r.force is None for r in done):
        raise RuntimeError("a request without a result")
    lat = np.array([r.done - r.arrival for r in done]) * 1e3
    return {"requests": len(done), "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
            "mean_ms": float(lat.mean()), "solves_per_s": len(done) / wall}


def make_requests(n, rate, n_bodies, seed=5):
    """Poisson arrivals: body index, omega U(0.1, 2.5), heading U(0, 180) deg."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, n)) if rate > 0 else np.zeros(n)
    idx = rng.integers(0, n_bodies, n)
    om = rng.uniform(0.1, 2.5, n)
    beta = rng.uniform(0.0, 180.0, n)
    return [Request(i, int(idx[i]), float(om[i]), float(beta[i]), float(t[i])) for i in range(n)]


def make_bodies(n_bodies, seed=5, n_min=200, n_max=3000):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n_bodies):
        mesh, depth = C.random_body(rng, n_min, n_max)
        out.append(Body(mesh, depth))
    return out
