"""Continuous-batching solve server on one GPU.

Requests are (body, omega, heading) solves of Nemoh's per-frequency BEM
problem: the diffraction problem at the request's heading plus the body's 6
radiation DOFs, i.e. one (mesh, omega) system with 7 right-hand sides, whose
result is the force matrix (nint x 7) of Solver/NEMOH.f90:137-141. The
reference has no server: it runs one body's frequencies one after another
(NEMOH.f90:129-143) with right-hand sides from its pre-processor
(preProcessor/BodyConditions.f90:27-137).

Design:
* resident bodies -- every body's mesh, generalised normals and DOFs are
  added to every worker's context once (nemoh_b200_add_body,
  nemoh_b200_set_body_dofs); a batch names bodies by index, nothing is
  uploaded per request but (omega, heading);
* right-hand sides on the device -- nemoh_b200_solve_requests builds each
  request's diffraction and radiation conditions with the pre-processor's
  formulas in a kernel;
* cross-body batches -- a batch holds requests of any bodies; their systems
  (of different orders) share one launch sequence (ragged batch);
* admission by HBM footprint -- a batch takes waiting requests in arrival
  order while their matrices and workspace (Body.bytes_per_frequency) fit
  the worker's share of device memory;
* continuous batching -- workers (one library context, CUDA stream and
  workspace each) take the next batch as soon as they are free, so requests
  that arrive while others are on the GPU join the next batch and batches of
  different workers overlap on the device.
"""
import collections
import dataclasses
import gc
import threading
import time
from typing import List, Optional

import numpy as np

from . import FP64, MIXED, Solver, set_autotune  # noqa: F401
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
    force: Optional[np.ndarray] = None   # (nint, 7): diffraction at the heading, then the 6 radiation DOFs
    error: Optional[str] = None          # set when the request's batch failed


class Body:
    """One body of the stream: mesh, environment, 6 DOFs about the origin."""

    def __init__(self, mesh: C.Mesh, depth: float, rho=1025.0, g=9.81):
        self.case = C.Case(mesh, np.array([1.0]), np.array([0.0]), C.six_dofs(), C.six_dofs(), rho=rho, g=g,
                           depth=depth)
        self.mesh = mesh

    @property
    def npanels(self):
        return self.mesh.npanels

    def bytes_per_frequency(self):
        """Device bytes of one request: D and S in FP64, the FP32 copy of D,
        and the right-hand-side workspace, per symmetry class."""
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
                 solver_factory=None, memory_bytes=None, max_batch=64, autotune=False):
        """Every worker's context holds every body, with the bodies' Rankine
        parts evaluated up front (Solver.prepare_bodies). autotune=False turns
        the triangular sweep's autotuning off for the process, so that no
        request waits on timing runs of a batch shape it meets first."""
        self.bodies = bodies
        self.device = device
        self.precision = precision
        self.nworkers = workers
        self.memory_fraction = memory_fraction
        self.max_batch = max_batch
        self._lock = threading.Condition()
        self._pending = collections.deque()
        self._done: List[Request] = []
        self._failed: List[Request] = []
        self._feeding = False
        make = solver_factory or (lambda: Solver(device, precision))
        self._solvers = [make() for _ in range(workers)]
        for s in self._solvers:
            for b in bodies:
                bid = s.add_body(b.case)
                s.set_body_dofs(bid, b.case.rad)
            if hasattr(s, "prepare_bodies"):
                s.prepare_bodies()
        if not autotune and solver_factory is None:
            set_autotune(False)
        self.batches = []   # (worker, bodies in the batch, nreq, t0, t1)
        free = memory_bytes
        if free is None:
            import torch
            free, _ = torch.cuda.mem_get_info(device)
        self._budget = free * memory_fraction / workers

    def close(self):
        for s in self._solvers:
            s.close()

    def admission(self, body: Body):
        """Requests of this body alone that fit a worker's share of HBM."""
        return max(1, int(self._budget // body.bytes_per_frequency()))

    def _take_batch(self):
        """Waiting requests in arrival order while they fit the budget (at least one)."""
        with self._lock:
            while not self._pending:
                if not self._feeding:
                    return None
                self._lock.wait(timeout=0.005)
            batch, used = [], 0
            while self._pending and len(batch) < self.max_batch:
                need = self.bodies[self._pending[0].body].bytes_per_frequency()
                if batch and used + need > self._budget:
                    break
                batch.append(self._pending.popleft())
                used += need
            return batch

    def _worker(self, w, t0):
        s = self._solvers[w]
        while True:
            batch = self._take_batch()
            if batch is None:
                return
            tb = time.perf_counter() - t0
            for r in batch:
                r.start = tb
            try:
                force = s.solve_requests(np.array([r.body for r in batch]), np.array([r.omega for r in batch]),
                                         np.radians([r.beta_deg for r in batch]))
            except Exception as e:   # the batch fails as a whole; the worker serves on
                td = time.perf_counter() - t0
                for r in batch:
                    r.error = "%s: %s" % (type(e).__name__, e)
                    r.done = td
                with self._lock:
                    self._failed.extend(batch)
                continue
            td = time.perf_counter() - t0
            for r, f in zip(batch, force):
                r.force = f
                r.done = td
            with self._lock:
                self._done.extend(batch)
                self.batches.append((w, len({r.body for r in batch}), len(batch), tb, td))

    def run(self, requests: List[Request], realtime=True):
        """Feed requests at their arrival times (or all at once) and wait for all results.

        Python's cyclic garbage collector is off while the stream runs (and back
        to the caller's setting after): its full collections over the server's
        request objects paused the workers and the feeder for tens to hundreds of
        ms, the largest part of the latency tails (requests and results are freed
        by reference counting regardless)."""
        gc_on = gc.isenabled()
        gc.disable()
        try:
            return self._run(requests, realtime)
        finally:
            if gc_on:
                gc.enable()

    def _run(self, requests: List[Request], realtime):
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
