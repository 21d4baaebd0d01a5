"""The C ABI: the library loads without a GPU and exports every declared symbol."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for h in os.listdir(os.path.join(ROOT, "include")):
        if h.endswith(".h"):
            text = open(os.path.join(ROOT, "include", h)).read()
            text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
            names |= set(re.findall(r"\b(btk_[a-z0-9_]+)\s*\(", text))
    return sorted(names)


def test_header_declares_the_reference_entry_points():
    names = declared_symbols()
    for ref in ("read_run_config", "tree_construction_2d", "tree_construction_3d", "dual_tree_traversal_2d",
                "dual_tree_traversal_3d", "split_interactions", "upward_pass_2d", "upward_pass_3d",
                "poisson_fmm_interactions_2d", "poisson_fmm_interactions_3d", "poisson_vel_fmm_interactions_3d",
                "downward_pass_2d", "downward_pass_3d", "downward_pass_3d_3"):
        assert "btk_" + ref in names


def test_library_exports_every_declared_symbol(lib):
    missing = [n for n in declared_symbols() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_covers_the_header():
    from barytreek_b200 import _lib
    assert set(declared_symbols()) <= set(_lib.SIGNATURES)


def test_struct_layouts_match_reference_sizes():
    from barytreek_b200 import _lib
    assert ctypes.sizeof(_lib.RunConfig) == 64
    assert ctypes.sizeof(_lib.TreeInfo) == 16
    assert _lib.PANEL2_DTYPE.itemsize == 80 and _lib.PANEL3_DTYPE.itemsize == 112
    assert _lib.PAIR_DTYPE.itemsize == 12
    assert _lib.RunConfig.ker_eps.offset == 48 and _lib.RunConfig.fmm_theta.offset == 16


def test_struct_layouts_match_reference_library(reflib):
    from barytreek_b200 import _lib
    sizes = [reflib.sizeof(i) for i in range(5)]
    assert sizes == [ctypes.sizeof(_lib.RunConfig), ctypes.sizeof(_lib.TreeInfo), _lib.PANEL2_DTYPE.itemsize,
                     _lib.PANEL3_DTYPE.itemsize, _lib.PAIR_DTYPE.itemsize]


def test_library_metadata(lib):
    assert lib.btk_version().startswith(b"barytreek_b200")
    assert lib.btk_max_degree() == 12
    assert lib.btk_launch_count() >= 0


def test_device_entry_points_validate_before_touching_the_device(lib):
    """Bad arguments are rejected with a status, not a crash (no GPU needed)."""
    from barytreek_b200 import _lib
    import barytreek_b200 as btk
    cfg = btk.make_run_config(3, 8, 100)
    ti = _lib.TreeInfo()
    st = lib.btk_upward_pass_3d(ctypes.byref(cfg), ctypes.byref(ti), None, None, None, None, None, None, None, 0, None)
    assert st == _lib.ERR_INVALID_ARGUMENT
    assert lib.btk_last_error()
    bad = btk.make_run_config(3, 13, 100)
    st = lib.btk_upward_pass_3d(ctypes.byref(bad), ctypes.byref(ti), None, None, None, None, None, None, None, 0, None)
    assert st == _lib.ERR_UNSUPPORTED
    st = lib.btk_direct_sum(2, 1, 0.0, 1, None, None, None, 1, None, None, None, None, None, None)
    assert st == _lib.ERR_INVALID_ARGUMENT
