"""The learned solve's audit and the interaction kernels' bounded waits.

* The audit is an FP64 direct sum: its relative L2 reading equals, to 1e-10,
  the relative L2 of the returned result against btk_direct_sum (FP64, the
  reference's direct sum, src/direct_sum_impl.hpp:34-94) on the same audited
  targets, for the mixed-precision learned solve (potential + gradient and the
  reference's vector kernel).
* The fallback decision is taken on that reading: with the degrees held fixed
  (a fixed per-pair tolerance), a tolerance 1e-6 (relative) below the audited
  error falls back to the plain FP64 result, one 1e-6 above it does not.
* Bounded waits: with the mbarrier poll limit at 0 every interaction block
  gives up at its first wait, drains its copies and leaves; the plain,
  mixed and learned solves then report BTK_ERR_DEVICE_TIMEOUT, and the next
  solve on the same plan (default limit) matches the oracle again.
* A plain per-pair solve after a learned solve on the same plan runs at the
  degrees set for the plan, not at the learned choice.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b)))


def direct_at(tc, q, kind, eps, idx):
    import torch
    from barytreek_b200 import _lib
    L = _lib.load()
    t = [torch.from_numpy(np.ascontiguousarray(c[idx])).cuda() for c in tc.targets]
    out = torch.empty((tc.ncomp, len(idx)), dtype=torch.float64, device="cuda")
    qd = torch.from_numpy(np.ascontiguousarray(q)).cuda()
    s = tc._s
    _lib.check(L.btk_direct_sum(3, kind, eps, len(idx), _lib.ptr(t[0]), _lib.ptr(t[1]), _lib.ptr(t[2]), tc.ns,
                                _lib.ptr(s[0]), _lib.ptr(s[1]), _lib.ptr(s[2]), _lib.ptr(qd), _lib.ptr(out), None))
    return out.cpu().numpy()


def learned_plan(pts, kind, eps, theta=0.7, leaf=500):
    import barytreek_b200 as btk
    return btk.Treecode(pts, degree=8, cluster_size=leaf, theta=theta, eps=eps, kind=kind,
                        precision=btk.PREC_MIXED, degree_mode=btk._lib.DEGREE_PER_PAIR, degree_min=4,
                        leaf_far_pairs=True)


def oracle_solve(oracle, tc, kind, q):
    t = tc.tree_t
    pp, pc, cp, cc = tc.lists
    tree = {"dim": 3, "degree": tc.cfg.interp_degree, "eps": tc.cfg.ker_eps, "thresh": tc.cfg.fmm_cluster_thresh,
            "targets": tc.targets, "sources": tc.targets, "panels_t": t.panels, "panels_s": t.panels,
            "level_start_t": t.level_start, "level_start_s": t.level_start, "leaf_of_s": t.point_leaf_panel,
            "inside_t": t.panel_points_inside, "inside_s": t.panel_points_inside, "pp": pp, "pc": pc, "cp": cp,
            "cc": cc}
    return oracle.solve(tree, kind, q)["out"]


@pytest.mark.parametrize("kind,eps,theta", [(2, 1e-4, 0.7), (1, 1e-3, 0.8)], ids=["field", "vel"])
def test_audit_reads_the_fp64_error(kind, eps, theta):
    from barytreek_b200 import datagen, selector
    pts, q = datagen.uniform_box(31, 120000, 3, 0.0, 1.0)
    tc = learned_plan(pts, kind, eps, theta)
    sel = selector.Selector.load(kind=kind)
    out, rep = tc.solve_learned(q, sel, tol=1e-6, pair_tol=1e-7)
    idx = tc.audit_targets()
    assert len(idx) == 1200 and rep["audit_targets"] == len(idx)
    ds = direct_at(tc, q, kind, eps, idx)
    e_true = rel(out.cpu().numpy()[:, idx], ds)
    assert 1e-9 < e_true < 1e-5
    assert abs(rep["audit_rel_l2"] - e_true) <= 1e-10, (rep["audit_rel_l2"], e_true)
    tc.close()


def test_fallback_decided_on_the_fp64_reading():
    import barytreek_b200 as btk
    from barytreek_b200 import datagen, selector
    pts, q = datagen.plummer(32, 100000)
    tc = learned_plan(pts, 2, 1e-4)
    sel = selector.Selector.load(kind=2)
    # the largest of these per-pair tolerances whose solve passes tol = 1e-6
    for pair_tol in (1e-7, 3e-8, 1e-8, 3e-9, 1e-9):
        out, rep = tc.solve_learned(q, sel, tol=1e-6, pair_tol=pair_tol)
        if rep["fell_back"] == 0:
            break
    e = rep["audit_rel_l2"]
    assert rep["fell_back"] == 0 and e > 0, rep
    out_hi, rep_hi = tc.solve_learned(q, sel, tol=e * (1 + 1e-6), pair_tol=pair_tol)
    assert rep_hi["fell_back"] == 0, (rep_hi["audit_rel_l2"], e)
    assert rel(out_hi.cpu().numpy(), out.cpu().numpy()) <= 1e-12
    out_lo, rep_lo = tc.solve_learned(q, sel, tol=e * (1 - 1e-6), pair_tol=pair_tol)
    assert rep_lo["fell_back"] == 1, (rep_lo["audit_rel_l2"], e)
    plain = btk.Treecode(pts, degree=8, cluster_size=500, theta=0.7, eps=1e-4, kind=2)
    assert rel(out_lo.cpu().numpy(), plain.solve(q).cpu().numpy()) <= 1e-12
    plain.close()
    tc.close()


@pytest.mark.parametrize("precision", [0, 1], ids=["fp64", "mixed"])
def test_wait_limit_timeout_then_recovery(oracle, precision):
    import barytreek_b200 as btk
    from barytreek_b200 import _lib, datagen
    pts, q = datagen.uniform_box(33, 4000, 3, 0.0, 1.0)
    tc = btk.Treecode(pts, degree=5, cluster_size=100, theta=0.7, eps=1e-4, kind=2, precision=precision)
    tc.set_wait_limit(0)
    tc.solve(q)
    with pytest.raises(_lib.BtkError) as ei:
        tc.last_timing()
    assert ei.value.status == _lib.ERR_DEVICE_TIMEOUT
    tc.set_wait_limit(-1)
    out = tc.solve(q).cpu().numpy()
    tc.last_timing()
    ref = oracle_solve(oracle, tc, 2, q)
    assert rel(out, ref) <= (1e-12 if precision == 0 else 1e-6)
    tc.close()


def test_wait_limit_timeout_in_learned_solve():
    from barytreek_b200 import _lib, datagen, selector
    pts, q = datagen.uniform_box(34, 30000, 3, 0.0, 1.0)
    tc = learned_plan(pts, 2, 1e-4, leaf=300)
    sel = selector.Selector.load(kind=2)
    ref, _ = tc.solve_learned(q, sel, tol=1e-6, pair_tol=1e-7)
    ref = ref.cpu().numpy()
    tc.set_wait_limit(0)
    with pytest.raises(_lib.BtkError) as ei:
        tc.solve_learned(q, sel, tol=1e-6, pair_tol=1e-7)
    assert ei.value.status == _lib.ERR_DEVICE_TIMEOUT
    tc.set_wait_limit(-1)
    out, rep = tc.solve_learned(q, sel, tol=1e-6, pair_tol=1e-7)
    assert rep["fell_back"] == 0
    assert rel(out.cpu().numpy(), ref) <= 1e-12
    tc.close()


def test_plain_solve_after_learned_uses_the_set_degrees(oracle):
    import barytreek_b200 as btk
    from barytreek_b200 import datagen, selector
    pts, q = datagen.uniform_box(35, 30000, 3, 0.0, 1.0)
    kw = dict(degree=8, cluster_size=300, theta=0.7, eps=1e-4, kind=2, precision=btk.PREC_FP64,
              degree_mode=btk._lib.DEGREE_PER_PAIR, degree_min=4, leaf_far_pairs=True)
    tc = btk.Treecode(pts, **kw)
    fresh = btk.Treecode(pts, **kw)
    st0 = tc.stats()
    sel = selector.Selector.load(kind=2)
    tc.solve_learned(q, sel, tol=1e-6, pair_tol=1e-6)
    out = tc.solve(q).cpu().numpy()
    assert rel(out, fresh.solve(q).cpu().numpy()) <= 1e-13
    assert tc.stats() == st0
    assert rel(out, oracle_solve(oracle, tc, 2, q)) <= 1e-12
    tc.close()
    fresh.close()
