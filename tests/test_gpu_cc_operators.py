"""The shared-matrix CC form (``cc_operators=True``) on the GPU.

CC pairs grouped by level and lattice offset are applied as one FP64 matrix
product per group; the result must match the oracle (the reference's pairwise
method) to the plain form's 1e-12, in every kind and in 2-D and 3-D, and the
pairwise plan to summation-order rounding at scale.
"""
import numpy as np
import pytest

from test_gpu_parity import CASES, make, rel, tree_dict

pytestmark = pytest.mark.gpu

TOL = 1e-12


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_cc_operators_match_oracle(case, oracle):
    import barytreek_b200 as btk
    _, dim, n, dist, deg, leaf, theta, eps, kind = case
    pts, _, q = make(dim, n, dist=dist)
    tc = btk.Treecode(pts, degree=deg, cluster_size=leaf, theta=theta, eps=eps, kind=kind, cc_operators=True)
    st = tc.stats()
    if len(tc.lists[3]):
        assert st["cc_groups"] > 0 and st["cc_tasks"] >= st["cc_groups"]
    out = tc.solve(q).cpu().numpy()
    ref = oracle.solve(tree_dict(tc), kind, q)["out"]
    for c in range(tc.ncomp):
        assert rel(out[c], ref[c]) <= TOL, (c, rel(out[c], ref[c]))


def test_cc_operators_against_reference_library(reflib):
    import barytreek_b200 as btk
    pts, _, q = make(3, 12000, seed=21)  # 1,672 CC pairs in 262 groups
    for kind in (0, 1):
        tc = btk.Treecode(pts, degree=6, cluster_size=150, theta=0.7, eps=1e-4, kind=kind, cc_operators=True)
        assert tc.stats()["cc_groups"] > 0
        out = tc.solve(q).cpu().numpy()
        rt = reflib.create(3, pts, degree=6, cluster_size=150, theta=0.7, eps=1e-4)
        ref = rt.solve(kind, q, fixed=True)["out"]
        for c in range(tc.ncomp):
            assert rel(out[c], ref[c]) <= TOL


@pytest.mark.parametrize("degree", [1, 4, 10, 12])
def test_cc_operators_degrees(degree, oracle):
    import barytreek_b200 as btk
    pts, _, q = make(3, 2500, seed=11)
    tc = btk.Treecode(pts, degree=degree, cluster_size=40, theta=0.7, eps=1e-4, kind=2, cc_operators=True)
    out = tc.solve(q).cpu().numpy()
    ref = oracle.solve(tree_dict(tc), 2, q)["out"]
    assert rel(out, ref) <= TOL


def test_cc_operators_eps_zero(oracle):
    """eps = 0: the guarded reciprocal path of the grouped kernel. Targets and
    sources are distinct point sets over the same root box [-1, 1]^3 (opposite
    corners in each), so the two trees group and no pair coincides."""
    import barytreek_b200 as btk
    rng = np.random.default_rng(9)
    t = np.vstack([[[-1, -1, -1], [1, 1, 1]], rng.uniform(-0.99, 0.99, (3000, 3))])
    s = np.vstack([[[-1, 1, 1], [1, -1, -1]], rng.uniform(-0.99, 0.99, (2500, 3))])
    pts, src = tuple(t.T.copy()), tuple(s.T.copy())
    q = rng.uniform(-1, 1, len(s))
    tc = btk.Treecode(pts, src, degree=5, cluster_size=30, theta=0.7, eps=0.0, kind=2, cc_operators=True)
    assert tc.stats()["cc_groups"] > 0
    out = tc.solve(q).cpu().numpy()
    ref = oracle.solve(tree_dict(tc), 2, q)["out"]
    assert rel(out, ref) <= TOL


def test_cc_operators_split_trees_fall_back_to_pairwise(oracle):
    """Source tree over another root box: no grouping, pairwise CC, same result."""
    import barytreek_b200 as btk
    pts, src, q = make(3, 3000, seed=5, ns=2500)
    tc = btk.Treecode(pts, src, degree=5, cluster_size=60, theta=0.7, eps=1e-4, kind=0, cc_operators=True)
    assert tc.stats()["cc_groups"] == 0
    out = tc.solve(q).cpu().numpy()
    ref = oracle.solve(tree_dict(tc), 0, q)["out"]
    assert rel(out, ref) <= TOL


@pytest.mark.parametrize("precision", [0, 1])
def test_cc_operators_at_scale(precision):
    """3-D potential + gradient, 262,144 uniform points, n = 8, leaf 500: the
    grouped form against the pairwise plan of the same precision (FP64: 1e-13;
    mixed: both within 1e-6 of each other), repeat solves identical to
    rounding, and the interaction phase faster than the pairwise one."""
    import torch

    import barytreek_b200 as btk
    from barytreek_b200 import datagen
    pts, q = datagen.uniform_box(2, 1 << 18, 3, 0.0, 1.0)
    qd = torch.from_numpy(q).cuda()
    kw = dict(degree=8, cluster_size=500, theta=0.7, eps=1e-4, kind=2, precision=precision)
    pair = btk.Treecode(pts, **kw)
    grp = btk.Treecode(pts, cc_operators=True, **kw)
    st = grp.stats()
    assert st["cc_groups"] > 0 and st["evals_cc"] == pair.stats()["evals_cc"]
    for _ in range(2):
        a = pair.solve(qd)
        torch.cuda.synchronize()
        ta = pair.last_timing()
        b = grp.solve(qd)
        torch.cuda.synchronize()
        tb = grp.last_timing()
    a, b = a.cpu().numpy(), b.cpu().numpy()
    assert rel(b, a) <= (1e-13 if precision == 0 else 1e-6)
    assert rel(grp.solve(qd).cpu().numpy(), b) <= 1e-14
    assert tb["interactions"] < ta["interactions"], (tb, ta)
