"""Well-separated leaf pairs in the learned degree choice (``leaf_far_pairs``).

Non-touching PP pairs within the separation bound (``leaf_far_theta``, default
0.8) may be approximated as target
points x source-leaf proxies at a chosen degree, or kept direct. With every
degree in force at the plan degree (btk_plan_execute) they are direct, so the
plan must reproduce the plan without them; learned solves must keep the
1e-6 accuracy against the FP64 direct sum, pass their audit without falling
back, and evaluate fewer pairs directly.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b)))


def _direct(tc, q, kind, eps, m=2000, seed=99):
    import torch
    from barytreek_b200 import _lib
    L = _lib.load()
    idx = np.sort(np.random.default_rng(seed).choice(tc.nt, m, replace=False))
    t = [torch.from_numpy(np.ascontiguousarray(c[idx])).cuda() for c in tc.targets]
    out = torch.empty((tc.ncomp, m), dtype=torch.float64, device="cuda")
    qd = torch.from_numpy(np.ascontiguousarray(q)).cuda()
    s = tc._s
    z = lambda a: _lib.ptr(a[2]) if tc.dim == 3 else None
    _lib.check(L.btk_direct_sum(tc.dim, kind, eps, m, _lib.ptr(t[0]), _lib.ptr(t[1]), z(t), tc.nt, _lib.ptr(s[0]),
                                _lib.ptr(s[1]), z(s), _lib.ptr(qd), _lib.ptr(out), None))
    return idx, out.cpu().numpy()


def test_degrees_in_force_keep_leaf_pairs_direct():
    import barytreek_b200 as btk
    from barytreek_b200 import _lib, datagen
    pts, q = datagen.uniform_box(3, 200_000, 3, 0.0, 1.0)
    kw = dict(degree=6, cluster_size=500, theta=0.7, eps=1e-4, kind=btk.KIND_FIELD, precision=btk.PREC_MIXED,
              degree_mode=_lib.DEGREE_PER_PAIR, degree_min=4)
    a = btk.Treecode(pts, **kw)
    b = btk.Treecode(pts, leaf_far_pairs=True, **kw)
    sb = b.stats()
    assert a.stats()["leaf_far_pairs"] == 0 and sb["leaf_far_pairs"] > 0
    assert sb["evals_pp"] == a.stats()["evals_pp"] and b.evals() == a.evals()
    ra, rb = a.solve(q).cpu().numpy(), b.solve(q).cpu().numpy()
    assert rel(rb, ra) <= 1e-14
    # the separation bound: the traversal's theta admits fewer pairs than the default 0.8
    c = btk.Treecode(pts, leaf_far_pairs=True, leaf_far_theta=0.7, **kw)
    assert 0 < c.stats()["leaf_far_pairs"] < sb["leaf_far_pairs"]
    assert rel(c.solve(q).cpu().numpy(), ra) <= 1e-14
    c.close()
    # per-list degrees leave the leaf pairs direct
    pc = len(b.lists[1])
    b.set_degrees(deg_pc=np.full(pc, 4, np.int32))
    a.set_degrees(deg_pc=np.full(pc, 4, np.int32))
    assert rel(b.solve(q).cpu().numpy(), a.solve(q).cpu().numpy()) <= 1e-14


@pytest.mark.parametrize("case", ["uniform-field-1m", "plummer-pot-1m", "mixture-field-262k"])
def test_learned_with_leaf_pairs(case):
    import torch

    import barytreek_b200 as btk
    from barytreek_b200 import _lib, datagen, selector
    if case == "uniform-field-1m":
        pts, q = datagen.uniform_box(1, 1 << 20, 3, 0.0, 1.0)
        kind, leaf, deg = btk.KIND_FIELD, 2000, 8
    elif case == "plummer-pot-1m":
        pts, q = datagen.plummer(2, 1 << 20)
        kind, leaf, deg = btk.KIND_POT, 2000, 8
    else:
        pts, q = datagen.gaussian_mixture(3, 1 << 18)
        kind, leaf, deg = btk.KIND_FIELD, 1000, 8
    qd = torch.from_numpy(q).cuda()
    kw = dict(degree=deg, cluster_size=leaf, theta=0.7, eps=1e-4, kind=kind, precision=btk.PREC_MIXED,
              degree_mode=_lib.DEGREE_PER_PAIR, degree_min=4)
    sel = selector.Selector.load(kind=kind)
    base = btk.Treecode(pts, **kw)
    for _ in range(3):
        _, rb = base.solve_learned(qd, sel, tol=1e-6)
    base.close()
    tc = btk.Treecode(pts, leaf_far_pairs=True, **kw)
    for _ in range(3):
        out, rep = tc.solve_learned(qd, sel, tol=1e-6)
    idx, ds = _direct(tc, q, kind, 1e-4)
    err = rel(out.cpu().numpy()[:, idx], ds)
    assert rep["fell_back"] == 0, rep
    assert rep["audit_rel_l2"] <= 1e-6
    assert err <= 1e-6, err
    assert rep["evals_near"] < rb["evals_near"]
    assert rep["ms_total"] < rb["ms_total"], (rep["ms_total"], rb["ms_total"])


@pytest.mark.parametrize("dim,kind,deg,leaf", [(3, 2, 5, 40), (3, 2, 2, 40), (3, 1, 2, 60), (2, 0, 2, 30),
                                               (2, 2, 4, 30)])
def test_leaf_forms_match_oracle(dim, kind, deg, leaf, oracle):
    """Forms and degrees set on every leaf pair (btk_plan_set_leaf_forms):
    direct, target points x source-leaf proxies, or proxies x proxies (the
    pairs whose target leaf exceeds the plan degree's proxies; at degree 2 the
    40-point leaves do). The plain FP64 solve must equal, to 1e-12, the oracle
    fed the same pairs as PP, PC (leaf source) and CC (leaf target and
    source) pairs at those degrees."""
    import ctypes

    import barytreek_b200 as btk
    from barytreek_b200 import _lib, datagen
    from test_gpu_degrees import tree_dict
    pts, q = datagen.uniform_box(4, 3000, dim, -1.0, 1.0)
    tc = btk.Treecode(pts, degree=deg, cluster_size=leaf, theta=0.7, eps=1e-4, kind=kind,
                      degree_mode=_lib.DEGREE_PER_PAIR, degree_min=2, leaf_far_pairs=True)
    L = _lib.load()
    n, ncc = ctypes.c_int(), ctypes.c_int()
    _lib.check(L.btk_plan_leaf_pairs(tc._plan, ctypes.byref(n), ctypes.byref(ncc), None))
    assert n.value > 0
    if deg == 2:
        assert ncc.value > 0
    idx = np.zeros(n.value, np.int32)
    _lib.check(L.btk_plan_leaf_pairs(tc._plan, ctypes.byref(n), ctypes.byref(ncc), _lib.ptr(idx)))
    rng = np.random.default_rng(3)
    form = rng.integers(0, 2, n.value).astype(np.int32)
    form[:ncc.value] = rng.integers(0, 3, ncc.value)
    dg = rng.integers(2, deg + 1, n.value).astype(np.int32)
    _lib.check(L.btk_plan_set_leaf_forms(tc._plan, _lib.ptr(form), _lib.ptr(dg)))
    out = tc.solve(q).cpu().numpy()
    pp, pc, cp, cc = tc.lists
    keep = np.ones(len(pp), bool)
    keep[idx[form != 0]] = False
    t = tree_dict(tc)
    t["pp"], t["pc"], t["cc"] = pp[keep], np.concatenate([pc, pp[idx[form == 1]]]), np.concatenate([cc, pp[idx[form == 2]]])
    d_pc = np.concatenate([np.full(len(pc), deg), dg[form == 1]]).astype(np.int32)
    d_cc = np.concatenate([np.full(len(cc), deg), dg[form == 2]]).astype(np.int32)
    ref = oracle.solve_degrees(t, kind, q, d_pc, np.full(len(cp), deg, np.int32), d_cc)
    for c in range(tc.ncomp):
        assert rel(out[c], ref[c]) <= 1e-12, (c, rel(out[c], ref[c]))
    # the PP count drops by the leaf pairs that left the direct form
    pts_t, pts_s = tc.tree_t.panels["point_count"], tc.tree_t.panels["point_count"]
    moved = pp[idx[form != 0]]
    st = tc.stats()
    assert st["evals_pp"] == int(sum(int(pts_t[a]) * int(pts_s[b]) for a, b in zip(pp["target_panel"][keep],
                                                                                     pp["source_panel"][keep])))
    assert len(moved) == int((form != 0).sum())
