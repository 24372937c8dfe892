"""Scheduling logic of the serving layer, with a fake solver (no GPU)."""
import threading
import time

import numpy as np

from nemoh_b200 import cases as C
from nemoh_b200 import serving as S


class FakeSolver:
    """Resident bodies; a request's forces are a fixed function of (body,
    omega, heading), the same alone and in any batch; records batch sizes."""
    calls = []
    lock = threading.Lock()

    def __init__(self):
        self.cases = []

    def add_body(self, case):
        self.cases.append(case)
        return len(self.cases) - 1

    def set_body_dofs(self, body, dofs):
        assert len(dofs) == 6

    def solve_requests(self, bodies, omegas, betas):
        time.sleep(0.002)
        with FakeSolver.lock:
            FakeSolver.calls.append(len(bodies))
        out = []
        for b, w, be in zip(bodies, omegas, betas):
            n = self.cases[b].mesh.npanels
            out.append(np.outer(np.arange(1, 7), np.arange(1, 8)) * (w + 1j * np.cos(be)) * n)
        return out

    def close(self):
        pass


def _bodies():
    return [S.Body(C.cylinder_mesh(3.0, 4.0, 8, 3, 2, 4), 0.0), S.Body(C.box_mesh(10, 6, 3, 4, 3, 2), 30.0)]


def test_every_request_served_once_and_batched():
    FakeSolver.calls = []
    bodies = _bodies()
    srv = S.SolveServer(bodies, workers=2, solver_factory=FakeSolver, memory_bytes=1 << 30)
    reqs = S.make_requests(60, rate=0, n_bodies=2, seed=1)
    done, wall = srv.run(reqs, realtime=False)
    assert sorted(r.rid for r in done) == list(range(60))
    assert max(FakeSolver.calls) > 1          # requests were batched
    for r in done:
        assert r.done >= r.start >= r.arrival


def test_result_same_alone_and_in_the_mix():
    bodies = _bodies()
    srv = S.SolveServer(bodies, workers=2, solver_factory=FakeSolver, memory_bytes=1 << 30)
    reqs = S.make_requests(40, rate=0, n_bodies=2, seed=2)
    done, _ = srv.run(reqs, realtime=False)
    alone, _ = srv.run([S.Request(99, reqs[7].body, reqs[7].omega, reqs[7].beta_deg)], realtime=False)
    mixed = {r.rid: r for r in done}[7]
    assert np.allclose(alone[0].force, mixed.force, rtol=1e-12, atol=0)


def test_admission_limits_batch_by_memory():
    FakeSolver.calls = []
    bodies = _bodies()
    budget = bodies[0].bytes_per_frequency() * 3 * 2 / 0.6   # 3 frequencies per worker
    srv = S.SolveServer(bodies[:1], workers=2, solver_factory=FakeSolver, memory_bytes=budget)
    assert srv.admission(bodies[0]) == 3
    reqs = [S.Request(i, 0, 0.5 + 0.01 * i, 0.0) for i in range(20)]
    done, _ = srv.run(reqs, realtime=False)
    assert len(done) == 20 and max(FakeSolver.calls) <= 3


class FailingSolver(FakeSolver):
    """Raises on every batch that contains the frequency 0.777 (a status-code error)."""

    def solve_requests(self, bodies, omegas, betas):
        if np.any(np.isclose(omegas, 0.777)):
            raise RuntimeError("nemoh_b200 status 5: EAKZ")
        return super().solve_requests(bodies, omegas, betas)


def test_failed_batch_is_reported_not_dropped():
    bodies = _bodies()
    srv = S.SolveServer(bodies, workers=2, solver_factory=FailingSolver, memory_bytes=1 << 30)
    reqs = S.make_requests(30, rate=0, n_bodies=2, seed=3)
    reqs[11].omega = 0.777
    try:
        srv.run(reqs, realtime=False)
    except S.ServeError as e:
        failed = {r.rid for r in e.failed}
        assert 11 in failed and all(r.error and "EAKZ" in r.error for r in e.failed)
        assert len(e.failed) + len(e.done) == 30          # every request accounted for
        assert not failed & {r.rid for r in e.done}
    else:
        raise AssertionError("a failed batch went unreported")
    # the server still serves afterwards, and the statistics check the count
    done, wall = srv.run(reqs[:5] + reqs[12:20], realtime=False)
    st = S.latency_stats(done, wall, expected=13)
    assert st["requests"] == 13
    try:
        S.latency_stats(done[:-1], wall, expected=13)
    except RuntimeError:
        pass
    else:
        raise AssertionError("a short result list went unnoticed")


def test_collector_off_during_a_stream_and_restored():
    """The cyclic garbage collector is off while a stream runs (its pauses were
    the latency tails) and back to the caller's setting afterwards, also when a
    batch fails."""
    import gc

    seen = []

    class Probe(FakeSolver):
        def solve_requests(self, bodies, omegas, betas):
            seen.append(gc.isenabled())
            return super().solve_requests(bodies, omegas, betas)

    srv = S.SolveServer(_bodies(), workers=1, solver_factory=Probe, memory_bytes=1 << 30)
    was = gc.isenabled()
    try:
        gc.enable()
        srv.run(S.make_requests(8, rate=0, n_bodies=2, seed=3), realtime=False)
        assert seen and not any(seen)
        assert gc.isenabled()
        gc.disable()
        srv.run(S.make_requests(4, rate=0, n_bodies=2, seed=4), realtime=False)
        assert not gc.isenabled()

        class Failing(FakeSolver):
            def solve_requests(self, bodies, omegas, betas):
                raise RuntimeError("planted failure")

        gc.enable()
        bad = S.SolveServer(_bodies(), workers=1, solver_factory=Failing, memory_bytes=1 << 30)
        try:
            bad.run(S.make_requests(3, rate=0, n_bodies=2, seed=5), realtime=False)
            raise AssertionError("a failed batch must raise")
        except S.ServeError:
            pass
        assert gc.isenabled()
    finally:
        if was:
            gc.enable()
        else:
            gc.disable()
