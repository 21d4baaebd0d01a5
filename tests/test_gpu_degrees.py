"""Per-pair interpolation degrees on the GPU (anterpolated source slots,
promoted target slots) against the oracle that evaluates every far-field pair
directly at its degree. Tolerance: relative L2 <= 1e-12 (FP64)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-12


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b)))


def tree_dict(tc):
    t = tc.tree_t
    s = tc.tree_s or tc.tree_t
    pp, pc, cp, cc = tc.lists
    return {"dim": tc.dim, "degree": tc.cfg.interp_degree, "eps": tc.cfg.ker_eps, "thresh": tc.cfg.fmm_cluster_thresh,
            "targets": tc.targets, "sources": tc.sources or tc.targets, "panels_t": t.panels, "panels_s": s.panels,
            "level_start_t": t.level_start, "level_start_s": s.level_start, "leaf_of_s": s.point_leaf_panel,
            "inside_t": t.panel_points_inside, "inside_s": s.panel_points_inside, "pp": pp, "pc": pc, "cp": cp,
            "cc": cc}


def problem(dim, n, dist, seed):
    from barytreek_b200 import datagen
    if dist == "plummer":
        return datagen.plummer(seed, n)
    if dist == "mixture":
        return datagen.gaussian_mixture(seed, n)
    return datagen.uniform_box(seed, n, dim, -1.0, 1.0)


@pytest.mark.parametrize("leaf_far", [False, True])
@pytest.mark.parametrize("dim,kind,dist,deg,leaf", [(3, 0, "plummer", 6, 60), (3, 2, "uniform", 5, 40),
                                                     (3, 1, "mixture", 6, 50), (2, 2, "uniform", 7, 30),
                                                     (2, 0, "uniform", 6, 40), (3, 2, "uniform", 2, 40),
                                                     (2, 2, "uniform", 2, 20)])
def test_random_degrees_match_oracle(dim, kind, dist, deg, leaf, leaf_far, oracle):
    """Set degrees: with leaf_far_pairs the plan also holds the leaf pairs and
    the proxy-to-proxy alternatives (at degree 2 the leaves exceed the plan
    degree's proxies, so every alternative exists); set_degrees keeps leaf pairs
    direct and every other pair in its own form, so the oracle is the same."""
    import barytreek_b200 as btk
    pts, q = problem(dim, 3000, dist, 5)
    tc = btk.Treecode(pts, degree=deg, cluster_size=leaf, theta=0.7, eps=1e-4, kind=kind,
                      degree_mode=btk._lib.DEGREE_PER_PAIR, degree_min=2, leaf_far_pairs=leaf_far)
    if leaf_far and deg == 2:
        assert tc.stats()["leaf_far_pairs"] > 0
    rng = np.random.default_rng(7)
    pp, pc, cp, cc = tc.lists
    assert len(pc) + len(cp) + len(cc) > 0
    d = [rng.integers(2, deg + 1, len(l)).astype(np.int32) for l in (pc, cp, cc)]
    tc.set_degrees(*d)
    out = tc.solve(q).cpu().numpy()
    ref = oracle.solve_degrees(tree_dict(tc), kind, q, *d)
    for c in range(tc.ncomp):
        assert rel(out[c], ref[c]) <= TOL, (c, rel(out[c], ref[c]))
    # work accounting follows the degrees
    s = tc.stats()
    m = lambda x: (x + 1) ** dim
    pts_t = tc.tree_t.panels["point_count"]
    assert s["evals_pc"] == sum(int(pts_t[p["target_panel"]]) * m(int(k)) for p, k in zip(pc, d[0]))
    assert s["evals_cc"] == sum(m(int(k)) ** 2 for k in d[2])


def test_per_pair_at_plan_degree_equals_fixed():
    import barytreek_b200 as btk
    pts, q = problem(3, 5000, "plummer", 9)
    kw = dict(degree=7, cluster_size=80, theta=0.7, eps=1e-4, kind=2)
    a = btk.Treecode(pts, **kw).solve(q).cpu().numpy()
    b = btk.Treecode(pts, degree_mode=btk._lib.DEGREE_PER_PAIR, degree_min=4, **kw).solve(q).cpu().numpy()
    assert rel(b, a) <= 1e-13


def test_per_pair_mixed_precision():
    import barytreek_b200 as btk
    pts, q = problem(3, 20000, "uniform", 11)
    kw = dict(degree=8, cluster_size=300, theta=0.7, eps=1e-4, kind=2, degree_mode=btk._lib.DEGREE_PER_PAIR,
              degree_min=3)
    rng = np.random.default_rng(3)
    a = btk.Treecode(pts, precision=btk.PREC_FP64, **kw)
    b = btk.Treecode(pts, precision=btk.PREC_MIXED, **kw)
    d = [rng.integers(3, 9, len(l)).astype(np.int32) for l in a.lists[1:]]
    a.set_degrees(*d)
    b.set_degrees(*d)
    ra, rb = a.solve(q).cpu().numpy(), b.solve(q).cpu().numpy()
    for c in range(ra.shape[0]):
        assert rel(rb[c], ra[c]) <= 5e-7


def test_degree_validation():
    import barytreek_b200 as btk
    pts, q = problem(3, 2000, "uniform", 13)
    tc = btk.Treecode(pts, degree=6, cluster_size=50, degree_mode=btk._lib.DEGREE_PER_PAIR, degree_min=3)
    with pytest.raises(btk.BtkError):
        tc.set_degrees(np.full(len(tc.lists[1]), 2, np.int32))
    fixed = btk.Treecode(pts, degree=6, cluster_size=50)
    with pytest.raises(btk.BtkError):
        fixed.set_degrees(np.full(len(fixed.lists[1]), 6, np.int32))
