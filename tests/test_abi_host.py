"""CPU checks of the product library: it builds, loads, exports the C-ABI,
and its host-side per-frequency setup equals the oracle's restatement of the
reference routines bit for bit (no GPU needed)."""
import math
import os
import re

import numpy as np
import pytest

import nemoh_b200 as nb
import oracle_lib as O
from nemoh_b200 import build as B

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module", autouse=True)
def built():
    B.build()


def _declared(header):
    txt = open(os.path.join(ROOT, "include", header)).read()
    return set(re.findall(r"\b(nemoh_b200_\w+)\s*\(", txt))


def test_library_exports_every_declared_symbol():
    L = nb.load_library()
    names = _declared("nemoh_b200.h") | _declared("nemoh_b200_diag.h")
    assert len(names) >= 16
    for n in names:
        assert hasattr(L, n), n


def test_create_without_device_fails_cleanly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    with pytest.raises(nb.NemohError) as e:
        nb.Solver()
    assert e.value.code == 22


@pytest.mark.parametrize("ak", [1e-3, 0.01, 0.1, 0.5, 1.0, 3.0, 10.0, 19.9])
def test_dispersion_root_bit_identical(ak):
    assert nb.dispersion_root(ak) == O.x0(ak)


def test_exponential_fit_bit_identical():
    n = 0
    for depth in (20.0, 50.0, 150.0):
        for w in np.linspace(0.05, 2.5, 40):
            akh0 = w * w * depth / 9.81
            if akh0 >= 20:
                continue
            amh = O.x0(akh0)
            akh = amh * math.tanh(amh)
            a = nb.exponential_fit(akh, amh)
            b = O.lisc(akh, amh)
            assert a[0] == b[0] and np.array_equal(a[1], b[1]) and np.array_equal(a[2], b[2]), (depth, w)
            n += 1
    assert n > 50


@pytest.mark.parametrize("akk", [0.1, 0.4, 0.41, 2.5, 3.0, 4.0, 5.0, 8.0, 9.0, 25.0, 26.0, 40.0, 41.0, 100.0])
def test_theta_quadrature_identical(akk):
    q1, c1 = nb.theta_quadrature(akk)
    q2, c2 = O.cint(akk)
    assert np.array_equal(q1, q2) and np.array_equal(c1, c2)


def test_stencil_thresholds_reproduce_truncation():
    kj8, kj5, ki5 = nb.stencil_thresholds()
    f8 = lambda x: int(8 * (math.log10(x) + 4.5))
    f5 = lambda x: int(5 * (math.log10(x) + 6))
    fi = lambda y: int(5 * (math.log10(y) + 6) + 1)
    rng = np.random.default_rng(1)
    cnt = lambda t, x: int(np.sum(x >= t)) - 1
    for x in 10 ** rng.uniform(-2, math.log10(16), 5000):
        assert max(min(cnt(kj8, x), 45), 2) == max(min(f8(x), 45), 2)
    for x in 10 ** rng.uniform(math.log10(1.5e-6), -2, 5000):
        assert max(min(cnt(kj5, x), 45), 2) == max(min(f5(x), 45), 2)
    for y in 10 ** rng.uniform(-20, 0, 5000):
        assert max(min(cnt(ki5, y), 327), 2) == max(min(fi(y), 327), 2)
    for t, f in ((kj8, f8), (kj5, f5), (ki5, fi)):
        for v in t:
            if np.isfinite(v) and v > 0:
                assert f(v) > f(np.nextafter(v, 0))
