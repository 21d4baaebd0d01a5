"""GPU parity: the CUDA path (through the C ABI) against the CPU oracle.

Tolerance for the plain FP64 form: relative L2 <= 1e-12 against the oracle
(the C restatement pinned to the reference, or the reference itself where its
library was built), on every output and intermediate the reference exposes.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-12


def rel(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


def tree_dict(tc):
    t = tc.tree_t
    s = tc.tree_s or tc.tree_t
    pp, pc, cp, cc = tc.lists
    return {"dim": tc.dim, "degree": tc.cfg.interp_degree, "eps": tc.cfg.ker_eps, "thresh": tc.cfg.fmm_cluster_thresh,
            "targets": tc.targets, "sources": tc.sources or tc.targets,
            "panels_t": t.panels, "panels_s": s.panels, "level_start_t": t.level_start,
            "level_start_s": s.level_start, "leaf_of_s": s.point_leaf_panel, "inside_t": t.panel_points_inside,
            "inside_s": s.panel_points_inside, "pp": pp, "pc": pc, "cp": cp, "cc": cc}


def make(dim, n, seed=1, dist="uniform", ns=None, **kw):
    from barytreek_b200 import datagen
    if dist == "uniform":
        pts, q = datagen.uniform_box(seed, n, dim, -1.0, 1.0)
    elif dist == "plummer":
        pts, q = datagen.plummer(seed, n)
    elif dist == "sphere":
        pts, q = datagen.sphere_surface(seed, n)
    else:
        pts, q = datagen.gaussian_mixture(seed, n)
    src = None
    if ns is not None:
        src, q = datagen.uniform_box(seed + 100, ns, dim, -1.0, 1.0)
    return pts, src, q


CASES = [
    # id, dim, n, dist, degree, leaf, theta, eps, kind
    ("2d-pot", 2, 3000, "uniform", 6, 60, 0.7, 1e-4, 0),
    ("2d-field", 2, 2500, "uniform", 5, 50, 0.7, 1e-4, 2),
    ("3d-pot", 3, 3000, "uniform", 5, 80, 0.7, 1e-4, 0),
    ("3d-vel", 3, 3000, "uniform", 5, 80, 0.7, 1e-4, 1),
    ("3d-field", 3, 3000, "uniform", 5, 80, 0.7, 1e-4, 2),
    ("3d-plummer-mixed-levels", 3, 4000, "plummer", 4, 300, 0.7, 1e-4, 0),
    ("3d-sphere-vel", 3, 3000, "sphere", 4, 100, 0.8, 1e-3, 1),
    ("3d-mixture-field", 3, 3000, "mixture", 4, 120, 0.6, 1e-4, 2),
]


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_plan_solve_matches_oracle(case, oracle):
    import barytreek_b200 as btk
    _, dim, n, dist, deg, leaf, theta, eps, kind = case
    pts, _, q = make(dim, n, dist=dist)
    tc = btk.Treecode(pts, degree=deg, cluster_size=leaf, theta=theta, eps=eps, kind=kind)
    out = tc.solve(q).cpu().numpy()
    ref = oracle.solve(tree_dict(tc), kind, q)["out"]
    for c in range(tc.ncomp):
        assert rel(out[c], ref[c]) <= TOL, (c, rel(out[c], ref[c]))


def test_split_trees_2d(oracle):
    import barytreek_b200 as btk
    pts, src, q = make(2, 2000, seed=5, ns=1500)
    tc = btk.Treecode(pts, src, degree=5, cluster_size=50, theta=0.7, eps=1e-4)
    out = tc.solve(q).cpu().numpy()
    ref = oracle.solve(tree_dict(tc), 0, q)["out"]
    assert rel(out, ref) <= TOL


def test_eps_zero_distinct_points(oracle):
    """eps = 0 takes the guarded reciprocal path (sources != targets)."""
    import barytreek_b200 as btk
    pts, src, q = make(3, 1500, seed=9, ns=1700)
    tc = btk.Treecode(pts, src, degree=4, cluster_size=60, theta=0.7, eps=0.0, kind=2)
    out = tc.solve(q).cpu().numpy()
    ref = oracle.solve(tree_dict(tc), 2, q)["out"]
    assert rel(out, ref) <= TOL


@pytest.mark.parametrize("degree", list(range(1, 13)))
def test_every_degree_3d(degree, oracle):
    import barytreek_b200 as btk
    pts, _, q = make(3, 1200, seed=11)
    tc = btk.Treecode(pts, degree=degree, cluster_size=40, theta=0.7, eps=1e-4)
    out = tc.solve(q).cpu().numpy()
    ref = oracle.solve(tree_dict(tc), 0, q)["out"]
    assert rel(out, ref) <= TOL


def test_against_reference_library(reflib):
    """Plan path vs the reference's own code (fixed downward), 3-D potential and velocity."""
    import barytreek_b200 as btk
    pts, _, q = make(3, 2500, seed=21, dist="plummer")
    for kind in (0, 1):
        tc = btk.Treecode(pts, degree=6, cluster_size=150, theta=0.7, eps=1e-4, kind=kind)
        out = tc.solve(q).cpu().numpy()
        rt = reflib.create(3, pts, degree=6, cluster_size=150, theta=0.7, eps=1e-4)
        ref = rt.solve(kind, q, fixed=True)["out"]
        for c in range(tc.ncomp):
            assert rel(out[c], ref[c]) <= TOL


def test_accuracy_vs_direct_sum(oracle):
    import barytreek_b200 as btk
    pts, _, q = make(3, 4000, seed=3)
    tc = btk.Treecode(pts, degree=8, cluster_size=100, theta=0.7, eps=1e-4, kind=2)
    out = tc.solve(q).cpu().numpy()
    ds = oracle.direct(3, 2, 1e-4, pts, pts, q)
    assert rel(out[0], ds[0]) < 1e-6
    assert rel(out[1:], ds[1:]) < 1e-5


@pytest.mark.parametrize("dim,kind", [(2, 0), (2, 2), (3, 0), (3, 1), (3, 2)])
def test_direct_sum_kernel(dim, kind, oracle, lib):
    import torch
    from barytreek_b200 import _lib
    pts, src, q = make(dim, 700, seed=31, ns=900)
    ref = oracle.direct(dim, kind, 1e-4, pts, src, q)
    dev = [torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in pts]
    sdev = [torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in src]
    qd = torch.from_numpy(q).cuda()
    nc = ref.shape[0]
    out = torch.empty((nc, len(pts[0])), dtype=torch.float64, device="cuda")
    z = _lib.ptr(dev[2]) if dim == 3 else None
    zs = _lib.ptr(sdev[2]) if dim == 3 else None
    _lib.check(lib.btk_direct_sum(dim, kind, 1e-4, len(pts[0]), _lib.ptr(dev[0]), _lib.ptr(dev[1]), z, len(src[0]),
                                  _lib.ptr(sdev[0]), _lib.ptr(sdev[1]), zs, _lib.ptr(qd), _lib.ptr(out), None))
    assert rel(out.cpu().numpy(), ref) <= 1e-13


def test_solve_host_matches_plan(lib):
    import barytreek_b200 as btk
    from barytreek_b200 import _lib
    pts, _, q = make(3, 3000, seed=41)
    tc = btk.Treecode(pts, degree=5, cluster_size=80, theta=0.7, eps=1e-4, kind=2)
    a = tc.solve(q).cpu().numpy()
    out = np.zeros((4, 3000))
    _lib.check(lib.btk_solve_host(3, 2, 0, 5, 80, 0.7, 1e-4, 3000, _lib.ptr(pts[0]), _lib.ptr(pts[1]),
                                  _lib.ptr(pts[2]), _lib.ptr(q), _lib.ptr(out), None))
    assert rel(out, a) <= 1e-14


def test_repeat_solves_are_identical():
    import barytreek_b200 as btk
    pts, _, q = make(3, 3000, seed=43)
    tc = btk.Treecode(pts, degree=6, cluster_size=80, theta=0.7, eps=1e-4)
    a = tc.solve(q).cpu().numpy()
    b = tc.solve(q).cpu().numpy()
    assert rel(a, b) <= 1e-15


# ---- drop-in entry points, phase by phase, against the reference functions ----

def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.mark.parametrize("dim,kind,dist", [(2, 0, "uniform"), (3, 0, "uniform"), (3, 1, "uniform"),
                                           (3, 0, "plummer")])
def test_dropin_phases(dim, kind, dist, oracle, lib):
    """upward_pass -> poisson_(vel_)fmm_interactions -> downward_pass through the
    reference-named C entry points on device arrays, each phase compared with
    the oracle's intermediate arrays."""
    import torch
    import barytreek_b200 as btk
    from barytreek_b200 import _lib
    pts, _, q = make(dim, 2500, seed=51, dist=dist)
    deg, leaf = (5, 70) if dim == 3 else (6, 50)
    cfg = btk.make_run_config(dim, deg, leaf, 0.7, 1e-4)
    tree = btk.tree_construction(cfg, pts)
    inter = btk.dual_tree_traversal(cfg, tree)
    lists = btk.split_interactions(cfg, inter)
    n, P, ipc = len(pts[0]), tree.panel_count, cfg.interp_point_count
    nc = 3 if kind == 1 else 1
    X = [_dev(a) for a in pts]
    Q = _dev(q)
    panels = _dev(tree.panels.view(np.uint8))
    leaf_of = _dev(tree.point_leaf_panel)
    inside = _dev(tree.panel_points_inside)
    L = [_dev(l.view(np.uint8)) if len(l) else None for l in lists]
    psw = torch.zeros((P, ipc), dtype=torch.float64, device="cuda")
    ptw = torch.zeros((nc, P, ipc), dtype=torch.float64, device="cuda")
    sol = torch.zeros((nc, n), dtype=torch.float64, device="cuda")
    ti = tree.tree_info()
    p = _lib.ptr
    Lp = [p(l) if l is not None else None for l in L]
    if dim == 2:
        _lib.check(lib.btk_upward_pass_2d(ctypes.byref(cfg), ctypes.byref(ti), p(X[0]), p(X[1]), p(Q), p(panels),
                                          p(psw), p(leaf_of), n, None))
    else:
        _lib.check(lib.btk_upward_pass_3d(ctypes.byref(cfg), ctypes.byref(ti), p(X[0]), p(X[1]), p(X[2]), p(Q),
                                          p(panels), p(psw), p(leaf_of), n, None))
    d = {"dim": dim, "degree": deg, "eps": 1e-4, "thresh": leaf, "targets": pts, "sources": pts,
         "panels_t": tree.panels, "panels_s": tree.panels, "level_start_t": tree.level_start,
         "level_start_s": tree.level_start, "leaf_of_s": tree.point_leaf_panel, "inside_t": tree.panel_points_inside,
         "inside_s": tree.panel_points_inside, "pp": lists[0], "pc": lists[1], "cp": lists[2], "cc": lists[3]}
    ref = oracle.solve(d, kind, q)
    assert rel(psw.cpu().numpy(), ref["psw"]) <= TOL
    if dim == 2:
        _lib.check(lib.btk_poisson_fmm_interactions_2d(
            ctypes.byref(cfg), p(X[0]), p(X[1]), p(X[0]), p(X[1]), p(Q), p(sol[0]), p(inside), p(inside), p(psw),
            p(ptw[0]), *Lp, p(panels), p(panels), n, n, P, P, None))
    elif kind == 0:
        _lib.check(lib.btk_poisson_fmm_interactions_3d(
            ctypes.byref(cfg), p(X[0]), p(X[1]), p(X[2]), p(X[0]), p(X[1]), p(X[2]), p(Q), p(sol[0]), p(inside),
            p(inside), p(psw), p(ptw[0]), *Lp, p(panels), p(panels), n, n, P, P, None))
    else:
        _lib.check(lib.btk_poisson_vel_fmm_interactions_3d(
            ctypes.byref(cfg), p(X[0]), p(X[1]), p(X[2]), p(X[0]), p(X[1]), p(X[2]), p(Q), p(sol[0]), p(sol[1]),
            p(sol[2]), p(inside), p(inside), p(psw), p(ptw[0]), p(ptw[1]), p(ptw[2]), *Lp, p(panels), p(panels),
            n, n, P, P, None))
    assert rel(sol.cpu().numpy(), ref["mid"]) <= TOL
    assert rel(ptw.cpu().numpy(), ref["ptw_mid"]) <= TOL
    if dim == 2:
        _lib.check(lib.btk_downward_pass_2d(ctypes.byref(cfg), ctypes.byref(ti), p(X[0]), p(X[1]), p(sol[0]),
                                            p(panels), p(ptw[0]), p(inside), n, None))
    elif kind == 0:
        _lib.check(lib.btk_downward_pass_3d(ctypes.byref(cfg), ctypes.byref(ti), p(X[0]), p(X[1]), p(X[2]),
                                            p(sol[0]), p(panels), p(ptw[0]), p(inside), n, None))
    else:
        _lib.check(lib.btk_downward_pass_3d_3(ctypes.byref(cfg), ctypes.byref(ti), p(X[0]), p(X[1]), p(X[2]),
                                              p(sol[0]), p(sol[1]), p(sol[2]), p(panels), p(ptw[0]), p(ptw[1]),
                                              p(ptw[2]), p(inside), n, None))
    assert rel(sol.cpu().numpy(), ref["out"]) <= TOL


def test_invalid_arguments_are_rejected(lib):
    import barytreek_b200 as btk
    from barytreek_b200 import _lib
    pts, _, q = make(3, 500, seed=61)
    with pytest.raises(btk.BtkError) as e:
        btk.Treecode(pts, degree=13, cluster_size=50)
    assert e.value.status == _lib.ERR_UNSUPPORTED
    with pytest.raises(btk.BtkError):
        btk.Treecode(pts, degree=4, cluster_size=50, kind=1, precision=7)


def _dropin_sequence(lib, cfg, ti, X, Q, panels, leaf_of, inside, L, n, P, ipc):
    """upward_pass_3d -> poisson_fmm_interactions_3d -> downward_pass_3d on
    fresh outputs; returns the potential."""
    import torch
    from barytreek_b200 import _lib
    p = _lib.ptr
    psw = torch.zeros((P, ipc), dtype=torch.float64, device="cuda")
    ptw = torch.zeros((P, ipc), dtype=torch.float64, device="cuda")
    sol = torch.zeros(n, dtype=torch.float64, device="cuda")
    Lp = [p(l) if l is not None else None for l in L]
    _lib.check(lib.btk_upward_pass_3d(ctypes.byref(cfg), ctypes.byref(ti), p(X[0]), p(X[1]), p(X[2]), p(Q),
                                      p(panels), p(psw), p(leaf_of), n, None))
    _lib.check(lib.btk_poisson_fmm_interactions_3d(
        ctypes.byref(cfg), p(X[0]), p(X[1]), p(X[2]), p(X[0]), p(X[1]), p(X[2]), p(Q), p(sol), p(inside), p(inside),
        p(psw), p(ptw), *Lp, p(panels), p(panels), n, n, P, P, None))
    _lib.check(lib.btk_downward_pass_3d(ctypes.byref(cfg), ctypes.byref(ti), p(X[0]), p(X[1]), p(X[2]), p(sol),
                                        p(panels), p(ptw), p(inside), n, None))
    return sol.cpu().numpy()


def test_dropin_cache_reuse_and_rebuild(oracle, lib):
    """The drop-in entry points keep what they derive from the caller's tree
    and lists between calls: a second call on the same buffers reuses it, and
    a tree rebuilt into the same buffers (points scaled by 1.25: the same
    counts and lists, other panel boxes) is detected and rebuilt. Each result
    matches the oracle to 1e-12."""
    import barytreek_b200 as btk
    pts, _, q = make(3, 3000, seed=52)
    cfg = btk.make_run_config(3, 5, 80, 0.7, 1e-4)
    results = []
    bufs = None
    for scale in (1.0, 1.0, 1.25):
        p_s = tuple(c * scale for c in pts)
        tree = btk.tree_construction(cfg, p_s)
        lists = btk.split_interactions(cfg, btk.dual_tree_traversal(cfg, tree))
        host = [tree.panels.view(np.uint8), tree.point_leaf_panel, tree.panel_points_inside] + \
               [l.view(np.uint8) for l in lists]
        if bufs is None:
            bufs = [_dev(a) for a in host]
        else:  # rebuilt into the same device buffers
            import torch
            for b, a in zip(bufs, host):
                assert b.numel() == a.size
                b.copy_(torch.from_numpy(np.ascontiguousarray(a)))
        X = [_dev(a) for a in p_s]
        out = _dropin_sequence(lib, cfg, tree.tree_info(), X, _dev(q), bufs[0], bufs[1], bufs[2], bufs[3:],
                               len(q), tree.panel_count, cfg.interp_point_count)
        d = {"dim": 3, "degree": 5, "eps": 1e-4, "thresh": 80, "targets": p_s, "sources": p_s,
             "panels_t": tree.panels, "panels_s": tree.panels, "level_start_t": tree.level_start,
             "level_start_s": tree.level_start, "leaf_of_s": tree.point_leaf_panel,
             "inside_t": tree.panel_points_inside, "inside_s": tree.panel_points_inside,
             "pp": lists[0], "pc": lists[1], "cp": lists[2], "cc": lists[3]}
        ref = oracle.solve(d, 0, q)["out"][0]
        assert rel(out, ref) <= TOL, scale
        results.append(out)
    assert rel(results[1], results[0]) <= 1e-14
