"""A request stream in small mixed-body batches, as a server issues it, with the
dataflow triangular sweep forced (NEMOH_B200_SWEEP is read once per process,
so the stream runs in a child process).

In such batches the systems' refinements converge at different passes, so the
later passes' sweeps skip the items of converged systems, many times over:
the path where a CTA claims its next item right after skipping one. Every
batch must succeed and every request's forces must match those of one FP64
call over the whole stream within 1e-6 of the request's largest force."""
import os
import subprocess
import sys

import numpy as np
import pytest

from nemoh_b200 import build as B

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))

SCRIPT = r"""
import sys, numpy as np
sys.path[:0] = [%r, %r]
import gpu_cases as G, nemoh_b200 as nb
from nemoh_b200 import cases as C
cases = list(G.small_cases())
rng = np.random.default_rng(21)
for _ in range(3):
    mesh, depth = C.random_body(rng, 150, 700)
    cases.append(C.Case(mesh, np.array([0.7]), np.array([0.0]), C.six_dofs(), C.six_dofs(), depth=depth))
rng = np.random.default_rng(5)
nb_batches = 400
sizes = rng.integers(1, 5, nb_batches)
body = rng.integers(0, len(cases), int(sizes.sum()))
omega = rng.uniform(0.3, 2.2, body.size)
beta = np.radians(rng.uniform(0.0, 180.0, body.size))
nb.set_autotune(False)
got = []
with nb.Solver(0, nb.MIXED) as s:
    for c in cases:
        s.set_body_dofs(s.add_body(c), c.rad)
    s.prepare_bodies()
    pos = 0
    for k in sizes:
        got += s.solve_requests(body[pos:pos + k], omega[pos:pos + k], beta[pos:pos + k])
        pos += k
    fb = s.fallback_count()
with nb.Solver(0, nb.FP64) as s:
    for c in cases:
        s.set_body_dofs(s.add_body(c), c.rad)
    ref = s.solve_requests(body, omega, beta)
worst = max(float(np.abs(g - r).max() / np.abs(r).max()) for g, r in zip(got, ref))
print("requests %%d batches %%d fallback %%s worst %%.3e" %% (body.size, nb_batches, fb, worst))
assert worst <= 1e-6, worst
"""


def test_request_stream_in_small_batches_with_the_dataflow_sweep(tmp_path):
    B.build()
    script = tmp_path / "stream.py"
    script.write_text(SCRIPT % (os.path.join(HERE, ".."), HERE))
    env = dict(os.environ, NEMOH_B200_SWEEP="flow")
    r = subprocess.run([sys.executable, str(script)], env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "worst" in r.stdout
