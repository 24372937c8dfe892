"""The synthetic meshes of the benchmark configurations (CPU)."""
import numpy as np

from nemoh_b200 import cases as C


def test_two_spheres_icosphere_mesh():
    """Precision configuration: two floating spheres R=4 m, centres 20 m apart,
    8,000 quad panels from quadrangulated icospheres, panel areas jittered by
    at most 10% from the seed."""
    case = C.config_two_spheres()
    m = case.mesh
    assert m.npanels == 8000 and m.nbodies == 2
    assert np.bincount(m.body)[1:].tolist() == [4000, 4000]
    assert m.nodes[:, 2].max() == 0.0 and m.nodes[:, 2].min() > -4.0
    xm, n, a = C.panel_quantities(m)
    # outward normals (the Solver's orientation) and the two centres
    centre = np.where(m.body[:, None] == 1, [-10.0, 0.0, 0.22], [10.0, 0.0, 0.22])
    assert np.all(np.einsum("ij,ij->i", n, xm - centre) > 0)
    # the hull area is that of the submerged cap (3.78 m draft) within the
    # discretisation error of flat panels
    cap = 2 * np.pi * 4.0 * 3.78
    assert abs(a[m.body == 1].sum() / cap - 1) < 0.03
    # the jitter changes areas by at most 10% against the unjittered hulls
    ref = [C.icosphere_hull(4.0, 12, -0.055, (c, 0.0), n_target=4000) for c in (-10.0, 10.0)]
    a0 = np.concatenate([C.panel_quantities(r)[2] for r in ref])
    ratio = a / a0
    assert ratio.min() >= 0.9 and ratio.max() <= 1.1
    assert ratio.max() - ratio.min() > 0.1          # and it does spread them
    # every panel's centroid below the free surface (the wave term is defined)
    assert xm[:, 2].max() < -1e-3


def test_icosphere_hull_counts():
    m = C.icosphere_hull(1.0, 6, 0.0)
    assert m.npanels % 3 == 0
    m2 = C.icosphere_hull(1.0, 6, 0.0, n_target=m.npanels + 5)
    assert m2.npanels == m.npanels + 5
