"""The learned degree selector on the GPU.

* BF16 MLP kernels (forward, gradient, Adam) against the FP64 numpy oracle on
  the same BF16-rounded weights; tolerance relative L2 <= 1e-4 (FP32 sums).
  The tensor-core inference against the oracle with BF16 activations (2e-3).
* Training samples (per-degree pair errors) against the CPU oracle evaluating
  the same single pair at the same degree and the direct sum; the log10 errors
  agree to 0.05 where the error is above 1e-11.
* The learned solve: the audit passes, the result meets the tolerance against
  the FP64 direct sum, and it needs fewer far-field evaluations than the fixed
  degree it replaces (the gain of the network); a forced failure falls back to
  the plain FP64 result.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b)))


@pytest.fixture(scope="module")
def batch():
    from oracle import mlp
    rng = np.random.default_rng(1)
    n = 300
    p = (rng.standard_normal(mlp.N_PARAMS) * 0.15).astype(np.float32)
    x = rng.standard_normal((n, mlp.F)).astype(np.float32)
    t = rng.standard_normal((n, mlp.O)).astype(np.float32)
    m = (rng.random((n, mlp.O)) > 0.2).astype(np.float32)
    return p, x, t, m


def test_mlp_forward_and_gradient_match_oracle(batch, lib):
    import torch
    from barytreek_b200 import _lib
    from oracle import mlp
    p, x, t, m = batch
    w = torch.from_numpy(p).cuda().to(torch.bfloat16)
    X, T, M = (torch.from_numpy(a).cuda() for a in (x, t, m))
    y = torch.empty_like(T)
    _lib.check(lib.btk_mlp_forward(_lib.ptr(w), len(x), _lib.ptr(X), _lib.ptr(y), None))
    pb = mlp.bf16_round(p)
    y_ref, _ = mlp.forward(pb, x.astype(np.float64))
    assert rel(y.cpu().numpy(), y_ref) <= 1e-4
    grad = torch.empty(mlp.N_PARAMS, dtype=torch.float32, device="cuda")
    loss = torch.zeros(1, dtype=torch.float32, device="cuda")
    work = torch.empty(len(x) * (4 * 64 + 9), dtype=torch.float32, device="cuda")
    _lib.check(lib.btk_mlp_gradient(_lib.ptr(w), len(x), _lib.ptr(X), _lib.ptr(T), _lib.ptr(M), _lib.ptr(grad),
                                    _lib.ptr(loss), _lib.ptr(work), None))
    l_ref, g_ref = mlp.loss_and_grad(pb, x.astype(np.float64), t.astype(np.float64), m.astype(np.float64))
    assert abs(loss.item() - l_ref) <= 1e-4 * abs(l_ref)
    assert rel(grad.cpu().numpy(), g_ref) <= 1e-4


def test_tensor_core_inference_matches_oracle(batch, lib):
    """btk_selector_predict (mma.sync BF16 products, FP32 sums, BF16-rounded
    inputs and activations) against the FP64 oracle of the same rounding:
    relative L2 <= 2e-3 (FP32 accumulation order and the rare activation whose
    BF16 rounding flips); against the FP32-activation forward kernel <= 2e-2.
    1,003 pairs: a partial 16-pair tile at the end, and a normalisation that
    shifts and scales every input and output."""
    import ctypes

    import torch
    from barytreek_b200 import _lib
    from oracle import mlp
    p, _, _, _ = batch
    rng = np.random.default_rng(7)
    n = 1003
    xm = rng.standard_normal(mlp.F).astype(np.float32)
    xs = (0.5 + rng.random(mlp.F)).astype(np.float32)
    norm = np.concatenate([xm, xs, [0.7, 1.9]]).astype(np.float32)
    feat = (xm + xs * rng.standard_normal((n, mlp.F))).astype(np.float32)
    sel = ctypes.c_void_p()
    _lib.check(lib.btk_selector_create(ctypes.byref(sel), _lib.ptr(p), _lib.ptr(norm)))
    try:
        F = torch.from_numpy(feat).cuda()
        out = torch.full((n, mlp.O), float("nan"), dtype=torch.float32, device="cuda")
        _lib.check(lib.btk_selector_predict(sel, n, _lib.ptr(F), _lib.ptr(out), None))
        torch.cuda.synchronize()
        got = out.cpu().numpy()
    finally:
        lib.btk_selector_destroy(sel)
    xn = (feat - xm) / xs
    pb = mlp.bf16_round(p)
    ref = mlp.forward_bf16_activations(pb, xn.astype(np.float32)) * 1.9 + 0.7
    assert np.isfinite(got).all()
    assert rel(got, ref) <= 2e-3
    ref32, _ = mlp.forward(pb, xn.astype(np.float64))
    assert rel(got, ref32 * 1.9 + 0.7) <= 2e-2


def test_adam_step_matches_oracle(batch, lib):
    import torch
    from barytreek_b200 import _lib
    from oracle import mlp
    p, x, t, m = batch
    rng = np.random.default_rng(2)
    g = (rng.standard_normal(mlp.N_PARAMS) * 0.01).astype(np.float32)
    master = torch.from_numpy(p.copy()).cuda()
    w = torch.empty(mlp.N_PARAMS, dtype=torch.bfloat16, device="cuda")
    mm = torch.zeros(mlp.N_PARAMS, dtype=torch.float32, device="cuda")
    vv = torch.zeros_like(mm)
    G = torch.from_numpy(g).cuda()
    ref_p, ref_m, ref_v = p.astype(np.float64), np.zeros(mlp.N_PARAMS), np.zeros(mlp.N_PARAMS)
    for step in (1, 2, 3):
        _lib.check(lib.btk_mlp_adam(_lib.ptr(master), _lib.ptr(w), _lib.ptr(G), _lib.ptr(mm), _lib.ptr(vv), step,
                                    ctypes.c_float(1e-3), None))
        ref_p, ref_m, ref_v = mlp.adam(ref_p, g.astype(np.float64), ref_m, ref_v, step, 1e-3)
    assert rel(master.cpu().numpy(), ref_p) <= 1e-6
    assert np.allclose(w.float().cpu().numpy(), mlp.bf16_round(master.cpu().numpy()), rtol=0, atol=0)


def _per_pair_tree(seed=3, n=6000, deg=8, leaf=150):
    import barytreek_b200 as btk
    from barytreek_b200 import datagen
    pts, q = datagen.plummer(seed, n)
    tc = btk.Treecode(pts, degree=deg, cluster_size=leaf, theta=0.7, eps=1e-4, kind=2,
                      degree_mode=btk._lib.DEGREE_PER_PAIR, degree_min=4)
    return tc, pts, q


def test_error_samples_match_oracle(oracle, lib):
    import torch
    from barytreek_b200 import _lib, selector
    tc, pts, q = _per_pair_tree(n=4000, deg=7, leaf=100)
    pp, pc, cp, cc = tc.lists
    lists = [("pc", pc), ("cp", cp), ("cc", cc)]
    rng = np.random.default_rng(9)
    K = 8
    picks = []  # (pair index in the PC,CP,CC order, class name, pair)
    off = 0
    for name, l in lists:
        for i in rng.choice(len(l), size=min(2, len(l)), replace=False):
            picks.append((off + int(i), name, l[i]))
        off += len(l)
    P = tc.tree_t.panels
    tgt_orig, csr, leaves = [], [0], []
    for _, _, pr in picks:
        lv = selector._subtree_leaves(P, int(pr["target_panel"]))
        pts_t = np.concatenate([tc.tree_t.panel_points_inside[l, :P["point_count"][l]] for l in lv])
        tgt_orig.append(pts_t[rng.integers(0, len(pts_t), K)])
        sl = selector._subtree_leaves(P, int(pr["source_panel"]))
        leaves += sl
        csr.append(len(leaves))
    tgt_orig = np.ascontiguousarray(np.array(tgt_orig), np.int32)
    csr, leaves = np.asarray(csr, np.int32), np.asarray(leaves, np.int32)
    pidx = np.asarray([p[0] for p in picks], np.int32)
    n_deg = 7 - 4 + 1
    out = np.zeros((len(picks), n_deg), np.float32)
    Q = torch.from_numpy(q).cuda()
    t, s = tc._t, tc._s
    _lib.check(lib.btk_plan_error_samples(tc._plan, _lib.ptr(t[0]), _lib.ptr(t[1]), _lib.ptr(t[2]), _lib.ptr(s[0]),
                                          _lib.ptr(s[1]), _lib.ptr(s[2]), _lib.ptr(Q), len(picks), _lib.ptr(pidx), K,
                                          _lib.ptr(tgt_orig), _lib.ptr(csr), _lib.ptr(leaves), None, _lib.ptr(out),
                                          None))
    base = {"dim": 3, "degree": 7, "eps": 1e-4, "thresh": 100, "targets": pts, "sources": pts, "panels_t": P,
            "panels_s": P, "level_start_t": tc.tree_t.level_start, "level_start_s": tc.tree_t.level_start,
            "leaf_of_s": tc.tree_t.point_leaf_panel, "inside_t": tc.tree_t.panel_points_inside,
            "inside_s": tc.tree_t.panel_points_inside}
    empty = np.zeros(0, pc.dtype)
    for j, (_, name, pr) in enumerate(picks):
        src_pts = np.concatenate([tc.tree_t.panel_points_inside[l, :P["point_count"][l]]
                                  for l in leaves[csr[j]:csr[j + 1]]])
        mask = np.zeros(len(q))
        mask[src_pts] = 1.0
        tg = tuple(c[tgt_orig[j]] for c in pts)
        exact = oracle.direct(3, 2, 1e-4, tg, pts, q * mask)
        for di, d in enumerate(range(4, 8)):
            tree = dict(base, pp=empty, pc=empty, cp=empty, cc=empty)
            tree[name] = np.array([pr], pc.dtype)
            approx = oracle.solve_degrees(tree, 2, q, np.full(1, d), np.full(1, d), np.full(1, d))[:, tgt_orig[j]]
            e_ref = np.log10(np.linalg.norm(approx - exact) / np.linalg.norm(exact) + 1e-30)
            if e_ref > -11:
                assert abs(out[j, di] - e_ref) <= 0.05, (name, d, out[j, di], e_ref)


def test_learned_solve_audit_gain_and_fallback(oracle):
    import barytreek_b200 as btk
    from barytreek_b200 import selector
    # train a small network on one problem, use it on another seed of the family
    tc, pts, q = _per_pair_tree(seed=3, n=20000, deg=8, leaf=200)
    X, E = selector.generate_samples(tc, q, n_samples=6000, K=16, seed=1)
    Y, M = selector.to_targets(E, 4, 8)
    sel = selector.train(X, Y, M, epochs=30, batch=512, lr=3e-3)
    tc2, pts2, q2 = _per_pair_tree(seed=4, n=20000, deg=8, leaf=200)
    tol = 1e-6
    out, rep = tc2.solve_learned(q2, sel, tol=tol, pair_tol=5e-8)
    out = out.cpu().numpy()
    assert rep["fell_back"] == 0, rep
    assert rep["audit_rel_l2"] <= tol
    ds = oracle.direct(3, 2, 1e-4, tuple(c[:400] for c in pts2), pts2, q2)
    assert rel(out[:, :400], ds) <= 2 * tol
    fixed = btk.Treecode(pts2, degree=8, cluster_size=200, theta=0.7, eps=1e-4, kind=2).stats()
    far_fixed = fixed["evals_pc"] + fixed["evals_cp"] + fixed["evals_cc"]
    assert rep["evals_far"] < 0.7 * far_fixed, (rep["evals_far"], far_fixed, rep["degree_hist"])
    # forced failure: every pair at degree 4 against a 1e-12 tolerance
    out2, rep2 = tc2.solve_learned(q2, sel, tol=1e-12, pair_tol=1.0)
    assert rep2["fell_back"] == 1
    plain = btk.Treecode(pts2, degree=8, cluster_size=200, theta=0.7, eps=1e-4, kind=2).solve(q2).cpu().numpy()
    assert rel(out2.cpu().numpy(), plain) <= 1e-12
