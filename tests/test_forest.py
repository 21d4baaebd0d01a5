"""Forest assembly for batches (host only, no GPU).

btk_forest_build builds every problem's tree and lists with the host tree
functions and renumbers the trees level-major into one panel array. Checked
here: mapping each forest panel back to (problem, local index) gives exactly
that problem's own tree (every field, with parent/children/id renumbered),
its own point_leaf_panel and its own four interaction lists in order; levels
are contiguous and level-major; counts add up; bad descriptors are rejected.
"""
import ctypes

import numpy as np
import pytest

from barytreek_b200 import _lib, datagen
from barytreek_b200.treecode import (PANEL2_DTYPE, PANEL3_DTYPE, dual_tree_traversal, make_run_config,
                                     split_interactions, tree_construction)


def _problems(dim, sizes, seed):
    out = []
    for b, n in enumerate(sizes):
        if dim == 3:
            pts, _ = datagen.gaussian_mixture(seed + b, n)
        else:
            pts, _ = datagen.uniform_box(seed + b, n, 2, -1.0, 1.0)
        out.append(pts)
    return out


def _build(lib, dim, probs, leaves, degree=4, theta=0.6, eps=1e-4):
    offs = np.zeros(len(probs) + 1, np.int32)
    offs[1:] = np.cumsum([len(p[0]) for p in probs])
    leaves = np.asarray(leaves, np.int32)
    xyz = [np.ascontiguousarray(np.concatenate([p[d] for p in probs])) for d in range(dim)]
    d = _lib.ForestDesc(dim, degree, theta, eps, len(probs), offs.ctypes.data, leaves.ctypes.data)
    f = _lib.Forest()
    st = lib.btk_forest_build(ctypes.byref(d), _lib.ptr(xyz[0]), _lib.ptr(xyz[1]),
                              _lib.ptr(xyz[2]) if dim == 3 else None, ctypes.byref(f))
    return st, f, offs, leaves


def _arr(addr, dtype, n):
    out = np.empty(n, dtype)
    if n:
        ctypes.memmove(out.ctypes.data, addr, out.nbytes)
    return out


@pytest.mark.parametrize("dim", [2, 3])
def test_forest_maps_back_to_each_problem(dim, lib):
    sizes = [3000, 700, 5200, 1, 2500] if dim == 3 else [4000, 900, 2600]
    probs = _problems(dim, sizes, 40 + dim)
    leaves = [200, 64, 500, 100, 150][:len(sizes)]
    st, f, offs, leaves = _build(lib, dim, probs, leaves)
    assert st == 0, lib.btk_last_error()
    try:
        P = f.info.panel_count
        pdt = PANEL3_DTYPE if dim == 3 else PANEL2_DTYPE
        panels = _arr(f.panels, pdt, P)
        ls = _arr(ctypes.cast(f.info.level_start, ctypes.c_void_p).value, np.int32, f.info.levels + 1)
        prob = _arr(f.panel_problem, np.int32, P)
        loc = _arr(f.panel_local, np.int32, P)
        leaf_of = _arr(f.point_leaf_panel, np.int32, offs[-1])
        lists = [_arr(getattr(f, n), _lib.PAIR_DTYPE, c) for n, c in
                 (("pp_list", f.cfg.fmm_pp_count), ("pc_list", f.cfg.fmm_pc_count), ("cp_list", f.cfg.fmm_cp_count),
                  ("cc_list", f.cfg.fmm_cc_count))]
        assert ls[0] == 0 and ls[-1] == P and np.all(np.diff(ls) >= 0)
        for l in range(f.info.levels):
            assert np.all(panels["level"][ls[l]:ls[l + 1]] == l)
        assert np.array_equal(panels["id"], np.arange(P))
        assert f.cfg.fmm_cluster_thresh == max(leaves)
        totals = [0, 0, 0, 0]
        for b, pts in enumerate(probs):
            cfg = make_run_config(dim, 4, int(leaves[b]), 0.6, 1e-4)
            tr = tree_construction(cfg, pts)
            own_lists = split_interactions(cfg, dual_tree_traversal(cfg, tr))
            mine = np.flatnonzero(prob == b)
            fwd = np.full(tr.panel_count, -1)
            fwd[loc[mine]] = mine
            assert np.all(fwd >= 0) and len(mine) == tr.panel_count
            fp = panels[fwd]
            for name in pdt.names:
                if name in ("id", "parent_id", "child"):
                    continue
                assert np.array_equal(fp[name], tr.panels[name]), (b, name)
            par = tr.panels["parent_id"]
            assert np.array_equal(fp["parent_id"], np.where(par >= 0, fwd[np.maximum(par, 0)], -1))
            ch = tr.panels["child"]
            assert np.array_equal(fp["child"], np.where(ch >= 0, fwd[np.maximum(ch, 0)], -1)), b
            assert np.array_equal(leaf_of[offs[b]:offs[b + 1]], fwd[tr.point_leaf_panel])
            for t in range(4):
                own = own_lists[t]
                got = lists[t][totals[t]:totals[t] + len(own)]
                totals[t] += len(own)
                assert np.array_equal(got["target_panel"], fwd[own["target_panel"]])
                assert np.array_equal(got["source_panel"], fwd[own["source_panel"]])
                assert np.array_equal(got["interact_type"], own["interact_type"])
        assert totals == [len(l) for l in lists]
    finally:
        lib.btk_forest_free(ctypes.byref(f))


def test_forest_rejects_bad_descriptors(lib):
    probs = _problems(3, [500, 400], 7)
    st, f, _, _ = _build(lib, 3, probs, [100, 0])
    assert st == _lib.ERR_INVALID_ARGUMENT and b"leaf sizes" in lib.btk_last_error()
    d = _lib.ForestDesc(3, 13, 0.6, 1e-4, 1, None, None)
    assert lib.btk_forest_build(ctypes.byref(d), None, None, None, ctypes.byref(_lib.Forest())) == \
        _lib.ERR_UNSUPPORTED


def test_autotuner_table_lookup():
    """Per-bucket lookup of the autotuner's table: leaf size by problem size,
    work split and tile size from the bucket holding most of a batch's points;
    two-entry tables (no tile) mean tiles of 256."""
    from barytreek_b200.batch import Autotuner
    t = Autotuner({12: (1024, 16, 256), 14: (512, 8, 128)})
    assert t.leaf_for(5000) == 1024 and t.leaf_for(20000) == 512 and t.leaf_for(9000) == 1024
    assert t.split_for_batch([5000] * 5 + [20000]) == 16 and t.tile_for_batch([5000] * 5 + [20000]) == 256
    assert t.split_for_batch([5000, 5000, 20000]) == 8 and t.tile_for_batch([5000, 5000, 20000]) == 128
    assert Autotuner({12: (1024, 16)}).tile_for_batch([5000]) == 256
