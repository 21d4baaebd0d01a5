"""Host tree functions: bit-identical to the reference (no GPU needed).

Trees, leaf lists, level starts, interaction lists and run configs are
compared field by field (padding bytes excluded) with the golden fixtures
produced by the reference, and with the reference library itself on further
seeded cases where it was built.
"""
import ctypes
import glob
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = sorted(glob.glob(os.path.join(HERE, "golden", "ref*.npz")))


def panels_equal(a, b):
    return all(np.array_equal(a[f], b[f]) for f in a.dtype.names)


def config_equal(cfg, raw_bytes):
    from barytreek_b200._lib import RunConfig
    rc = RunConfig.from_buffer_copy(bytes(raw_bytes))
    return all(getattr(cfg, f) == getattr(rc, f) for f, _ in cfg._fields_)


def build(dim, pts, deg, leaf, theta, eps, src=None):
    import barytreek_b200 as btk
    cfg = btk.make_run_config(dim, deg, leaf, theta, eps)
    tt = btk.tree_construction(cfg, pts)
    ts = btk.tree_construction(cfg, src) if src is not None else None
    inter = btk.dual_tree_traversal(cfg, tt, ts)
    lists = btk.split_interactions(cfg, inter)
    return cfg, tt, ts, inter, lists


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[:-4] for p in GOLDEN])
def test_tree_and_lists_match_golden(path):
    from barytreek_b200._lib import PANEL2_DTYPE, PANEL3_DTYPE, PAIR_DTYPE
    z = np.load(path)
    dim, n, seed, deg, leaf, ns = (int(v) for v in z["params"])
    theta, eps = (float(v) for v in z["fparams"])
    pts = tuple(z[f"t{d}"] for d in range(dim))
    src = tuple(z[f"s{d}"] for d in range(dim)) if ns else None
    cfg, tt, ts, inter, lists = build(dim, pts, deg, leaf, theta, eps, src)
    pdt = PANEL2_DTYPE if dim == 2 else PANEL3_DTYPE
    for tag, tr in (("T", tt), ("S", ts)):
        if tr is None:
            continue
        assert panels_equal(tr.panels, z[f"{tag}_panels"].view(pdt))
        assert np.array_equal(tr.level_start, z[f"{tag}_level_start"])
        assert np.array_equal(tr.point_leaf_panel, z[f"{tag}_leaf_of"])
        assert np.array_equal(tr.panel_points_inside, z[f"{tag}_inside"])
    assert np.array_equal(inter, z["all"].view(PAIR_DTYPE))
    for k, l in zip(("pp", "pc", "cp", "cc"), lists):
        assert np.array_equal(l, z[k].view(PAIR_DTYPE))
    assert config_equal(cfg, z["config"])


@pytest.mark.parametrize("name", ["nl_default", "nl_clamp", "nl_partial", "nl_eof"])
def test_read_run_config_matches_reference(name):
    import barytreek_b200 as btk
    z = np.load(os.path.join(HERE, "golden", name + ".npz"))
    for dim in (2, 3):
        cfg = btk.read_run_config(os.path.join(HERE, "golden", name + ".txt"), dim)
        ref = btk._lib.RunConfig.from_buffer_copy(bytes(z[f"cfg{dim}"]))
        # fields the reader sets (the rest is uninitialised in the reference)
        fields = ["dim", "fmm_theta"]
        text = open(os.path.join(HERE, "golden", name + ".txt")).read()
        if "interp_degree" in text.split("foo")[0]:
            fields += ["interp_degree", "interp_point_count"]
        if "cluster_size" in text:
            fields += ["fmm_cluster_thresh"]
        if "kernel_eps" in text:
            fields += ["ker_eps"]
        for f in fields:
            assert getattr(cfg, f) == getattr(ref, f), (name, dim, f)


def test_read_run_config_missing_file():
    import barytreek_b200 as btk
    with pytest.raises(btk.BtkError) as e:
        btk.read_run_config("/nonexistent/namelist.txt", 3)
    assert e.value.status == btk._lib.ERR_IO


def test_namelist_without_final_newline_terminates(tmp_path):
    """The reference re-parses the last line forever here; this reader stops."""
    import barytreek_b200 as btk
    p = tmp_path / "nl.txt"
    p.write_text("interp_degree=6\ncluster_size=50\ntheta=0.5")
    cfg = btk.read_run_config(str(p), 3)
    assert (cfg.interp_degree, cfg.interp_point_count, cfg.fmm_cluster_thresh, cfg.fmm_theta) == (6, 343, 50, 0.5)


def test_coincident_points_are_rejected():
    import barytreek_b200 as btk
    pts = (np.zeros(20), np.zeros(20), np.zeros(20))
    cfg = btk.make_run_config(3, 4, 5, 0.7, 1e-4)
    with pytest.raises(btk.BtkError):
        btk.tree_construction(cfg, pts)


def test_single_point_and_tiny_trees():
    import barytreek_b200 as btk
    for n in (1, 2, 7):
        pts = tuple(np.linspace(0, 1, n) * (d + 1) for d in range(3))
        cfg, tt, _, inter, lists = build(3, pts, 4, 10, 0.7, 1e-4)
        assert tt.panel_count == 1 and tt.levels == 1
        assert len(inter) == 1 and len(lists[0]) == 1  # the root-root PP pair


@pytest.mark.parametrize("seed,dim,n,dist,deg,leaf,theta", [
    (11, 3, 30000, "uniform", 8, 200, 0.7),
    (12, 3, 30000, "plummer", 6, 300, 0.6),
    (13, 3, 20000, "sphere", 5, 150, 0.8),
    (14, 3, 20000, "mixture", 6, 120, 0.6),
    (15, 2, 40000, "uniform", 8, 100, 0.7),
])
def test_against_reference_library(seed, dim, n, dist, deg, leaf, theta, reflib):
    from barytreek_b200 import datagen
    gen = {"uniform": lambda: datagen.uniform_box(seed, n, dim, -1, 1), "plummer": lambda: datagen.plummer(seed, n),
           "sphere": lambda: datagen.sphere_surface(seed, n), "mixture": lambda: datagen.gaussian_mixture(seed, n)}
    pts, q = gen[dist]()
    rt = reflib.create(dim, pts, degree=deg, cluster_size=leaf, theta=theta, eps=1e-4)
    cfg, tt, _, inter, lists = build(dim, pts, deg, leaf, theta, 1e-4)
    r = rt.trees[0]
    assert panels_equal(tt.panels, r["panels"])
    assert np.array_equal(tt.level_start, r["level_start"])
    assert np.array_equal(tt.point_leaf_panel, r["leaf_of"])
    assert np.array_equal(tt.panel_points_inside, r["inside"])
    assert np.array_equal(inter, rt.all)
    for k, l in zip(("pp", "pc", "cp", "cc"), lists):
        assert np.array_equal(l, rt.lists[k])
    assert config_equal(cfg, np.frombuffer(rt.config_bytes, np.uint8))
