"""Mixed precision (FP32 bulk on cluster-relative coordinates, compensated FP64
per-target sums) against the FP64 form and the FP64 direct sum.

Tolerances: relative L2 <= 5e-7 against the plain FP64 treecode on the same
tree (the FP32 evaluation error), and <= 1e-6 against the FP64 direct sum at
degree 8 (the accuracy target of the mixed form).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b)))


@pytest.mark.parametrize("dim,kind,dist", [(3, 0, "uniform"), (3, 2, "uniform"), (3, 1, "sphere"),
                                           (3, 2, "plummer"), (2, 0, "uniform"), (2, 2, "uniform")])
def test_mixed_matches_fp64(dim, kind, dist):
    import barytreek_b200 as btk
    from barytreek_b200 import datagen
    if dist == "uniform":
        pts, q = datagen.uniform_box(17, 20000, dim, -1.0, 1.0)
    elif dist == "sphere":
        pts, q = datagen.sphere_surface(17, 20000)
    else:
        pts, q = datagen.plummer(17, 20000)
    kw = dict(degree=7, cluster_size=300, theta=0.7, eps=1e-4, kind=kind)
    a = btk.Treecode(pts, precision=btk.PREC_FP64, **kw).solve(q).cpu().numpy()
    b = btk.Treecode(pts, precision=btk.PREC_MIXED, **kw).solve(q).cpu().numpy()
    for c in range(a.shape[0]):
        assert rel(b[c], a[c]) <= 5e-7, (c, rel(b[c], a[c]))


def test_mixed_accuracy_vs_direct_sum(oracle):
    import barytreek_b200 as btk
    from barytreek_b200 import datagen
    pts, q = datagen.uniform_box(19, 6000, 3, 0.0, 1.0)
    tc = btk.Treecode(pts, degree=8, cluster_size=200, theta=0.7, eps=1e-4, kind=2, precision=btk.PREC_MIXED)
    out = tc.solve(q).cpu().numpy()
    ds = oracle.direct(3, 2, 1e-4, pts, pts, q)
    assert rel(out, ds) <= 1e-6


def test_mixed_split_sources_eps_zero():
    import barytreek_b200 as btk
    from barytreek_b200 import datagen
    t, _ = datagen.uniform_box(23, 5000, 3, 0.0, 1.0)
    s, q = datagen.uniform_box(24, 7000, 3, 0.0, 1.0)
    kw = dict(degree=6, cluster_size=150, theta=0.7, eps=0.0, kind=0)
    a = btk.Treecode(t, s, precision=btk.PREC_FP64, **kw).solve(q).cpu().numpy()
    b = btk.Treecode(t, s, precision=btk.PREC_MIXED, **kw).solve(q).cpu().numpy()
    assert rel(b, a) <= 5e-7
