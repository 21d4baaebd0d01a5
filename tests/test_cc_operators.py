"""Host-side grouping of the CC list for the shared-matrix CC form.

Pairs grouped together must have the same target level, source level and
box-centre offset (so the same proxy-to-proxy matrix), pairs in different
groups must differ in one of them, and trees that are not subdivisions of one
common root box must not be grouped. Restated here with numpy from the panel
bounds (tree construction splits at midpoints: src/tree_construction.cpp:131-305).
"""
import numpy as np

from barytreek_b200 import datagen
from barytreek_b200 import treecode as T


def _centres(panels, dim):
    axes = ("x", "y", "z")[:dim]
    return np.stack([0.5 * (panels["min_" + a] + panels["max_" + a]) for a in axes], 1)


def _widths(panels, dim):
    axes = ("x", "y", "z")[:dim]
    return np.stack([panels["max_" + a] - panels["min_" + a] for a in axes], 1)


def _keys(dim, tt, cc, ts=None):
    ts = ts or tt
    ct, cs = _centres(tt.panels, dim), _centres(ts.panels, dim)
    root = tt.panels[0]
    w = _widths(tt.panels[:1], dim)[0]
    finest = max(tt.panels["level"].max(), ts.panels["level"].max())
    unit = np.where(w > 0, w / 2.0 ** (finest + 1), 1.0)
    lo = np.array([root["min_" + a] for a in ("x", "y", "z")[:dim]])
    it = np.rint((ct - lo) / unit).astype(np.int64)
    is_ = np.rint((cs - lo) / unit).astype(np.int64)
    t, s = cc["target_panel"], cc["source_panel"]
    return np.column_stack([tt.panels["level"][t], ts.panels["level"][s], it[t] - is_[s]]), ct[t] - cs[s]


def _check_grouping(dim, tt, cc, ts=None):
    g, n = T.cc_operator_groups(dim, tt, cc, ts)
    assert n > 0 and g.min() == 0 and g.max() == n - 1
    key, off = _keys(dim, tt, cc, ts)
    uk, inv = np.unique(key, axis=0, return_inverse=True)
    assert len(uk) == n
    # same key <=> same group (ids follow key order)
    assert np.array_equal(g, inv.ravel().astype(np.int32))
    # one group's pairs have the same centre offset to rounding
    for k in range(n):
        o = off[g == k]
        assert np.abs(o - o[0]).max() <= 1e-12 * max(1.0, np.abs(o[0]).max())
    return g, n


def test_groups_3d_uniform():
    pts, _ = datagen.uniform_box(3, 200_000, 3, 0.0, 1.0)
    cfg = T.make_run_config(3, 8, 500, 0.7)
    tr = T.tree_construction(cfg, pts)
    cc = T.split_interactions(cfg, T.dual_tree_traversal(cfg, tr))[3]
    assert len(cc) > 1000
    g, n = _check_grouping(3, tr, cc)
    assert n < len(cc) / 4  # translation invariance: many pairs per group


def test_groups_3d_plummer_and_2d():
    pts, _ = datagen.plummer(4, 100_000)
    cfg = T.make_run_config(3, 6, 300, 0.7)
    tr = T.tree_construction(cfg, pts)
    _check_grouping(3, tr, T.split_interactions(cfg, T.dual_tree_traversal(cfg, tr))[3])
    p2, _ = datagen.uniform_box(5, 65_536, 2, -1.0, 1.0)
    cfg2 = T.make_run_config(2, 8, 100, 0.7)
    t2 = T.tree_construction(cfg2, p2)
    _check_grouping(2, t2, T.split_interactions(cfg2, T.dual_tree_traversal(cfg2, t2))[3])


def test_split_trees_same_root_box_group_and_other_boxes_do_not():
    rng = np.random.default_rng(6)
    corners = np.array([[0, 0, 0], [1, 1, 1]], np.float64)
    a = np.vstack([corners, rng.random((60_000, 3))])
    b = np.vstack([corners, rng.random((50_000, 3)) ** 2])
    cfg = T.make_run_config(3, 6, 300, 0.7)
    ta = T.tree_construction(cfg, tuple(a.T.copy()))
    tb = T.tree_construction(cfg, tuple(b.T.copy()))
    cc = T.split_interactions(cfg, T.dual_tree_traversal(cfg, ta, tb))[3]
    assert len(cc) > 0
    _check_grouping(3, ta, cc, tb)
    # a source tree over another root box: no grouping
    c = np.vstack([corners * 1.5, rng.random((50_000, 3))])
    tc = T.tree_construction(cfg, tuple(c.T.copy()))
    cc2 = T.split_interactions(cfg, T.dual_tree_traversal(cfg, ta, tc))[3]
    g, n = T.cc_operator_groups(3, ta, cc2, tc)
    assert n == 0 and (len(g) == 0 or g.max() == -1)


def test_empty_cc_list():
    pts, _ = datagen.uniform_box(7, 1000, 3, 0.0, 1.0)
    cfg = T.make_run_config(3, 4, 2000, 0.7)
    tr = T.tree_construction(cfg, pts)
    g, n = T.cc_operator_groups(3, tr, np.zeros(0, T.PAIR_DTYPE))
    assert n == 0 and len(g) == 0
