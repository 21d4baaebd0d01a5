"""Device tree construction against the host tree functions (which the CPU
tests pin to the reference): every panel field, the level starts,
point_leaf_panel and the leaf rows must be identical, for 2-D and 3-D, several
distributions and leaf sizes up to 4M points, all-negative coordinates (the
reference's max() starting value), signed zeros at the extremes, NaN
coordinates, an empty input, a single leaf, and the coincident-points error.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _device_tree(lib, cfg, pts):
    import torch
    from barytreek_b200 import _lib
    from barytreek_b200.treecode import PANEL2_DTYPE, PANEL3_DTYPE, _copy_out
    dim = len(pts)
    n = len(pts[0])
    d = [torch.from_numpy(np.ascontiguousarray(c, np.float64)).cuda() for c in pts]
    leaf_of = torch.full((max(n, 1),), -7, dtype=torch.int32, device="cuda")
    order = torch.full((max(n, 1),), -7, dtype=torch.int32, device="cuda")
    info = _lib.TreeInfo()
    panels_p = ctypes.c_void_p()
    if dim == 3:
        st = lib.btk_tree_construction_3d_device(ctypes.byref(cfg), ctypes.byref(info), _lib.ptr(d[0]), _lib.ptr(d[1]),
                                                 _lib.ptr(d[2]), n, ctypes.byref(panels_p), _lib.ptr(leaf_of),
                                                 _lib.ptr(order), None)
    else:
        st = lib.btk_tree_construction_2d_device(ctypes.byref(cfg), ctypes.byref(info), _lib.ptr(d[0]), _lib.ptr(d[1]),
                                                 n, ctypes.byref(panels_p), _lib.ptr(leaf_of), _lib.ptr(order), None)
    if st != 0:
        return st, None
    try:
        panels = _copy_out(panels_p.value, PANEL2_DTYPE if dim == 2 else PANEL3_DTYPE, info.panel_count)
        ls = _copy_out(ctypes.cast(info.level_start, ctypes.c_void_p).value, np.int32, info.levels + 1)
    finally:
        lib.btk_free(panels_p)
        lib.btk_free(ctypes.cast(info.level_start, ctypes.c_void_p))
    return 0, (panels, ls, leaf_of.cpu().numpy()[:n], order.cpu().numpy()[:n])


def _compare(lib, dim, pts, leaf, degree=6):
    from barytreek_b200.treecode import make_run_config, tree_construction
    cfg = make_run_config(dim, degree, leaf, 0.7, 1e-4)
    host = tree_construction(cfg, pts)
    st, dev = _device_tree(lib, cfg, pts)
    assert st == 0, lib.btk_last_error()
    panels, ls, leaf_of, order = dev
    assert np.array_equal(ls, host.level_start)
    assert len(panels) == len(host.panels)
    for name in panels.dtype.names:
        a, b = panels[name], host.panels[name]
        if a.dtype.kind == "f":
            assert np.array_equal(a.view(np.uint64), b.view(np.uint64)), name  # bit-identical
        else:
            assert np.array_equal(a, b), name
    assert np.array_equal(leaf_of, host.point_leaf_panel)
    P = host.panels
    rows = [host.panel_points_inside[i, :P["point_count"][i]] for i in range(len(P))
            if P["is_leaf"][i] and P["point_count"][i] > 0]
    expect = np.concatenate(rows) if rows else np.zeros(0, np.int32)
    assert np.array_equal(order, expect)


@pytest.mark.parametrize("dim,dist,n,leaf", [(3, "uniform", 200000, 500), (3, "plummer", 300000, 300),
                                             (3, "sphere", 150000, 1000), (3, "mixture", 250000, 64),
                                             (2, "uniform", 100000, 200), (2, "uniform", 65536, 500),
                                             (3, "plummer", 1 << 22, 2000)])
def test_device_tree_matches_host(dim, dist, n, leaf, lib):
    from barytreek_b200 import datagen
    gen = {"uniform": lambda: datagen.uniform_box(3, n, dim, -1.0, 1.0)[0],
           "plummer": lambda: datagen.plummer(3, n)[0], "sphere": lambda: datagen.sphere_surface(3, n)[0],
           "mixture": lambda: datagen.gaussian_mixture(3, n)[0]}
    _compare(lib, dim, gen[dist](), leaf)


def test_device_tree_edge_cases(lib):
    from barytreek_b200 import datagen
    rng = np.random.default_rng(4)
    # all coordinates negative: the root's max stays at the smallest positive double
    pts = tuple(-1.0 - rng.random(5000) for _ in range(3))
    _compare(lib, 3, pts, 100)
    # signed zeros as extremes, in both orders
    for first in (0.0, -0.0):
        x = np.abs(rng.random(3000))
        x[10], x[20] = first, -first
        y = -np.abs(rng.random(3000))
        y[5], y[7] = -first, first
        _compare(lib, 3, (x, y, rng.random(3000)), 50)
    # NaN coordinates never set the box and fall in the lower halves
    x = rng.random(4000)
    x[[3, 99, 1500]] = np.nan
    _compare(lib, 2, (x, rng.random(4000)), 80)
    # empty input and a single leaf
    _compare(lib, 3, tuple(np.zeros(0) for _ in range(3)), 10)
    _compare(lib, 3, datagen.uniform_box(5, 90, 3, 0.0, 1.0)[0], 100)


def test_device_tree_rejects_coincident_points(lib):
    import torch
    from barytreek_b200 import _lib
    from barytreek_b200.treecode import make_run_config
    cfg = make_run_config(3, 4, 10, 0.7, 1e-4)
    pts = [torch.full((50,), 0.25, dtype=torch.float64, device="cuda") for _ in range(3)]
    leaf_of = torch.empty(50, dtype=torch.int32, device="cuda")
    info = _lib.TreeInfo()
    p = ctypes.c_void_p()
    st = lib.btk_tree_construction_3d_device(ctypes.byref(cfg), ctypes.byref(info), _lib.ptr(pts[0]), _lib.ptr(pts[1]),
                                             _lib.ptr(pts[2]), 50, ctypes.byref(p), _lib.ptr(leaf_of), None, None)
    assert st == _lib.ERR_INVALID_ARGUMENT and b"coincident" in lib.btk_last_error()


def test_treecode_on_device_tree_solves_alike():
    import time

    import barytreek_b200 as btk
    from barytreek_b200 import datagen
    pts, q = datagen.plummer(8, 400000)
    kw = dict(degree=7, cluster_size=1000, theta=0.7, eps=1e-4, kind=btk.KIND_FIELD)
    t0 = time.perf_counter()
    a = btk.Treecode(pts, **kw)
    t1 = time.perf_counter()
    b = btk.Treecode(pts, device_tree=True, **kw)
    t2 = time.perf_counter()
    for x, y in zip(a.lists, b.lists):
        assert np.array_equal(x, y)
    oa, ob = a.solve(q).cpu().numpy(), b.solve(q).cpu().numpy()
    assert np.linalg.norm(oa - ob) <= 1e-14 * np.linalg.norm(oa)
    print(f"plan set-up: host tree {t1 - t0:.3f} s, device tree {t2 - t1:.3f} s")


@pytest.mark.parametrize("dim,dist,n,leaf,theta,split", [(3, "uniform", 1 << 20, 2000, 0.7, False),
                                                         (3, "plummer", 1 << 22, 2000, 0.7, False),
                                                         (3, "sphere", 300000, 500, 0.8, False),
                                                         (3, "mixture", 200000, 100, 0.6, True),
                                                         (2, "uniform", 65536, 500, 0.7, False),
                                                         (2, "uniform", 50000, 60, 0.5, True)])
def test_device_traversal_matches_host(dim, dist, n, leaf, theta, split):
    from barytreek_b200 import datagen
    from barytreek_b200.treecode import (dual_tree_traversal, dual_tree_traversal_device, make_run_config,
                                         tree_construction)
    gen = {"uniform": lambda s, m: datagen.uniform_box(s, m, dim, -1.0, 1.0)[0],
           "plummer": lambda s, m: datagen.plummer(s, m)[0], "sphere": lambda s, m: datagen.sphere_surface(s, m)[0],
           "mixture": lambda s, m: datagen.gaussian_mixture(s, m)[0]}
    cfg_h = make_run_config(dim, 6, leaf, theta, 1e-4)
    cfg_d = make_run_config(dim, 6, leaf, theta, 1e-4)
    tt = tree_construction(cfg_h, gen[dist](3, n))
    ts = tree_construction(cfg_h, gen[dist](4, n // 2)) if split else None
    host = dual_tree_traversal(cfg_h, tt, ts)
    dev = dual_tree_traversal_device(cfg_d, tt, ts)
    assert np.array_equal(host, dev)
    for f in ("fmm_interaction_count", "fmm_pp_count", "fmm_pc_count", "fmm_cp_count", "fmm_cc_count"):
        assert getattr(cfg_h, f) == getattr(cfg_d, f), f
