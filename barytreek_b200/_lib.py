"""ctypes binding of the C ABI declared in include/barytreek_b200.h.

The shared library is built in-tree (``barytreek_b200/build.py``). Loading
fails loudly when it is missing: there is no CPU fallback for the device path.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libbarytreek_b200.so")

# Status codes (btk_status).
OK, ERR_INVALID_ARGUMENT, ERR_CUDA, ERR_UNSUPPORTED, ERR_OUT_OF_MEMORY, ERR_DEVICE_TIMEOUT, ERR_IO, ERR_INTERNAL = range(8)
KIND_POT, KIND_VEL, KIND_FIELD = 0, 1, 2
PREC_FP64, PREC_MIXED = 0, 1
DEGREE_RULE_THRESHOLD, DEGREE_RULE_COST = 0, 1
DEGREE_FIXED, DEGREE_PER_PAIR = 0, 1

# Reference struct layouts (src/structs.hpp), as numpy dtypes for host arrays.
PANEL2_DTYPE = np.dtype({
    "names": ["id", "level", "parent_id", "child", "is_leaf", "max_x", "min_x", "max_y", "min_y", "radius",
              "point_count"],
    "formats": ["<i4", "<i4", "<i4", ("<i4", 4), "u1", "<f8", "<f8", "<f8", "<f8", "<f8", "<i4"],
    "offsets": [0, 4, 8, 12, 28, 32, 40, 48, 56, 64, 72],
    "itemsize": 80,
})
PANEL3_DTYPE = np.dtype({
    "names": ["id", "level", "parent_id", "child", "is_leaf", "max_x", "min_x", "max_y", "min_y", "min_z", "max_z",
              "radius", "point_count"],
    "formats": ["<i4", "<i4", "<i4", ("<i4", 8), "u1", "<f8", "<f8", "<f8", "<f8", "<f8", "<f8", "<f8", "<i4"],
    "offsets": [0, 4, 8, 12, 44, 48, 56, 64, 72, 80, 88, 96, 104],
    "itemsize": 112,
})
PAIR_DTYPE = np.dtype([("target_panel", "<i4"), ("source_panel", "<i4"), ("interact_type", "<i4")])


class RunConfig(ctypes.Structure):
    """btk_run_config == RunConfig (src/structs.hpp:6-22)."""
    _fields_ = [("dim", ctypes.c_int), ("interp_degree", ctypes.c_int), ("interp_point_count", ctypes.c_int),
                ("fmm_theta", ctypes.c_double), ("fmm_cluster_thresh", ctypes.c_int),
                ("fmm_interaction_count", ctypes.c_int), ("fmm_pp_count", ctypes.c_int),
                ("fmm_pc_count", ctypes.c_int), ("fmm_cp_count", ctypes.c_int), ("fmm_cc_count", ctypes.c_int),
                ("ker_eps", ctypes.c_double), ("mpi_p", ctypes.c_int), ("mpi_id", ctypes.c_int)]


class TreeInfo(ctypes.Structure):
    """btk_tree_info == TreeInfo (src/structs.hpp:24-28)."""
    _fields_ = [("panel_count", ctypes.c_int), ("levels", ctypes.c_int), ("level_start", ctypes.POINTER(ctypes.c_int))]


class PlanDesc(ctypes.Structure):
    _fields_ = [("cfg", RunConfig), ("point_count_target", ctypes.c_int), ("point_count_source", ctypes.c_int),
                ("tree_target", ctypes.POINTER(TreeInfo)), ("tree_source", ctypes.POINTER(TreeInfo)),
                ("panels_target", ctypes.c_void_p), ("panels_source", ctypes.c_void_p),
                ("panel_points_inside_target", ctypes.c_void_p), ("panel_points_inside_source", ctypes.c_void_p),
                ("point_leaf_panel_source", ctypes.c_void_p), ("pp_list", ctypes.c_void_p),
                ("pc_list", ctypes.c_void_p), ("cp_list", ctypes.c_void_p), ("cc_list", ctypes.c_void_p),
                ("kind", ctypes.c_int), ("precision", ctypes.c_int), ("degree_mode", ctypes.c_int),
                ("degree_min", ctypes.c_int), ("work_split", ctypes.c_int), ("cc_operators", ctypes.c_int),
                ("leaf_far_pairs", ctypes.c_int), ("leaf_far_theta", ctypes.c_double),
                ("tile_targets", ctypes.c_int)]


class PlanStats(ctypes.Structure):
    _fields_ = [("evals_pp", ctypes.c_int64), ("evals_pc", ctypes.c_int64), ("evals_cp", ctypes.c_int64),
                ("evals_cc", ctypes.c_int64), ("work_items", ctypes.c_int64), ("device_bytes", ctypes.c_int64),
                ("levels_target", ctypes.c_int), ("levels_source", ctypes.c_int),
                ("build_ms_total", ctypes.c_float), ("build_ms_work", ctypes.c_float), ("cc_groups", ctypes.c_int),
                ("cc_tasks", ctypes.c_int), ("leaf_far_pairs", ctypes.c_int)]


class ForestDesc(ctypes.Structure):
    _fields_ = [("dim", ctypes.c_int), ("degree", ctypes.c_int), ("theta", ctypes.c_double), ("eps", ctypes.c_double),
                ("n_problems", ctypes.c_int), ("point_offset", ctypes.c_void_p), ("cluster_size", ctypes.c_void_p)]


class Forest(ctypes.Structure):
    _fields_ = [("cfg", RunConfig), ("info", TreeInfo), ("panels", ctypes.c_void_p),
                ("point_leaf_panel", ctypes.c_void_p), ("panel_problem", ctypes.c_void_p),
                ("panel_local", ctypes.c_void_p), ("pp_list", ctypes.c_void_p), ("pc_list", ctypes.c_void_p),
                ("cp_list", ctypes.c_void_p), ("cc_list", ctypes.c_void_p)]


class BatchDesc(ctypes.Structure):
    _fields_ = [("forest", ForestDesc), ("kind", ctypes.c_int), ("precision", ctypes.c_int),
                ("work_split", ctypes.c_int), ("tile_targets", ctypes.c_int)]


class BatchStats(ctypes.Structure):
    _fields_ = [("n_problems", ctypes.c_int), ("total_points", ctypes.c_int64), ("panel_count", ctypes.c_int),
                ("levels", ctypes.c_int), ("evals_pp", ctypes.c_int64), ("evals_pc", ctypes.c_int64),
                ("evals_cp", ctypes.c_int64), ("evals_cc", ctypes.c_int64), ("work_items", ctypes.c_int64),
                ("graph_kernel_nodes", ctypes.c_int), ("graph_nodes", ctypes.c_int), ("last_ms", ctypes.c_float)]


class BtkError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"btk status {status}: {msg}")
        self.status = status


_vp, _ci, _cd = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
_PRC = ctypes.POINTER(RunConfig)
_PTI = ctypes.POINTER(TreeInfo)

# name -> argtypes (restype btk_status/int unless listed in _RESTYPES)
SIGNATURES = {
    "btk_last_error": [],
    "btk_version": [],
    "btk_launch_count": [],
    "btk_max_degree": [],
    "btk_free": [_vp],
    "btk_read_run_config": [ctypes.c_char_p, _PRC],
    "btk_tree_construction_2d": [_PRC, _PTI, _vp, _vp, _ci, _vp, _vp, _vp],
    "btk_tree_construction_3d": [_PRC, _PTI, _vp, _vp, _vp, _ci, _vp, _vp, _vp],
    "btk_tree_construction_2d_device": [_PRC, _PTI, _vp, _vp, _ci, _vp, _vp, _vp, _vp],
    "btk_tree_construction_3d_device": [_PRC, _PTI, _vp, _vp, _vp, _ci, _vp, _vp, _vp, _vp],
    "btk_dual_tree_traversal_2d": [_PRC, _vp, _vp, _vp],
    "btk_dual_tree_traversal_3d": [_PRC, _vp, _vp, _vp],
    "btk_dual_tree_traversal_2d_device": [_PRC, _vp, _ci, _vp, _ci, _vp, _vp],
    "btk_dual_tree_traversal_3d_device": [_PRC, _vp, _ci, _vp, _ci, _vp, _vp],
    "btk_split_interactions": [_vp, _ci, _vp, _vp, _vp, _vp],
    "btk_upward_pass_2d": [_PRC, _PTI, _vp, _vp, _vp, _vp, _vp, _vp, _ci, _vp],
    "btk_upward_pass_3d": [_PRC, _PTI, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _ci, _vp],
    "btk_poisson_fmm_interactions_2d": [_PRC] + [_vp] * 16 + [_ci] * 4 + [_vp],
    "btk_poisson_fmm_interactions_3d": [_PRC] + [_vp] * 18 + [_ci] * 4 + [_vp],
    "btk_poisson_vel_fmm_interactions_3d": [_PRC] + [_vp] * 22 + [_ci] * 4 + [_vp],
    "btk_downward_pass_2d": [_PRC, _PTI, _vp, _vp, _vp, _vp, _vp, _vp, _ci, _vp],
    "btk_downward_pass_3d": [_PRC, _PTI, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _ci, _vp],
    "btk_downward_pass_3d_3": [_PRC, _PTI, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _ci, _vp],
    "btk_direct_sum": [_ci, _ci, _cd, _ci, _vp, _vp, _vp, _ci, _vp, _vp, _vp, _vp, _vp, _vp],
    "btk_direct_sum_noalloc": [_ci, _ci, _cd, _ci, _vp, _vp, _vp, _ci, _vp, _vp, _vp, _vp, _vp, _vp],
    "btk_plan_create": [_vp, ctypes.POINTER(PlanDesc), _vp],
    "btk_plan_destroy": [_vp],
    "btk_plan_stats_get": [_vp, ctypes.POINTER(PlanStats)],
    "btk_cc_operator_groups": [_ci, _vp, _ci, _vp, _ci, _vp, _ci, _vp, _vp],
    "btk_plan_execute": [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp],
    "btk_plan_last_timing": [_vp, _vp],
    "btk_dropin_cache_clear": [],
    "btk_plan_set_wait_limit": [_vp, ctypes.c_longlong],
    "btk_plan_audit_targets": [_vp, _vp, _vp],
    "btk_solve_host": [_ci, _ci, _ci, _ci, _ci, _cd, _cd, _ci, _vp, _vp, _vp, _vp, _vp, _vp],
    "btk_measure_pipe_peak": [_ci, _vp, _vp],
    "btk_plan_set_degrees": [_vp, _vp, _vp, _vp],
    "btk_plan_set_degree_rule": [_vp, _ci],
    "btk_selector_param_count": [],
    "btk_selector_create": [_vp, _vp, _vp],
    "btk_selector_destroy": [_vp],
    "btk_selector_weights": [_vp],
    "btk_plan_pair_count": [_vp, _vp],
    "btk_plan_leaf_pairs": [_vp, _vp, _vp, _vp],
    "btk_plan_set_leaf_forms": [_vp, _vp, _vp],
    "btk_selector_predict": [_vp, _ci, _vp, _vp, _vp],
    "btk_plan_pair_features": [_vp, _vp, _vp, _vp, _vp, _vp, _vp],
    "btk_plan_execute_learned": [_vp, _vp, _cd, _cd, _ci, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp],
    "btk_plan_error_samples": [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _ci, _vp, _ci, _vp, _vp, _vp, _vp, _vp, _vp],
    "btk_mlp_forward": [_vp, _ci, _vp, _vp, _vp],
    "btk_mlp_gradient": [_vp, _ci, _vp, _vp, _vp, _vp, _vp, _vp, _vp],
    "btk_mlp_adam": [_vp, _vp, _vp, _vp, _vp, _ci, ctypes.c_float, _vp],
    "btk_forest_build": [ctypes.POINTER(ForestDesc), _vp, _vp, _vp, ctypes.POINTER(Forest)],
    "btk_forest_free": [ctypes.POINTER(Forest)],
    "btk_batch_create": [_vp, ctypes.POINTER(BatchDesc), _vp, _vp, _vp, _vp],
    "btk_batch_destroy": [_vp],
    "btk_batch_execute": [_vp, _vp, _vp, _vp],
    "btk_batch_stats_get": [_vp, ctypes.POINTER(BatchStats)],
}
_RESTYPES = {"btk_last_error": ctypes.c_char_p, "btk_version": ctypes.c_char_p, "btk_launch_count": ctypes.c_uint64,
             "btk_free": None, "btk_selector_weights": ctypes.c_void_p, "btk_forest_free": None}


class LearnedReport(ctypes.Structure):
    """btk_learned_report."""
    _fields_ = [("audit_rel_l2", ctypes.c_double), ("audit_targets", ctypes.c_int), ("fell_back", ctypes.c_int),
                ("evals_near", ctypes.c_int64), ("evals_far", ctypes.c_int64), ("ms_select", ctypes.c_float),
                ("ms_solve", ctypes.c_float), ("ms_total", ctypes.c_float), ("degree_hist", ctypes.c_int * 13),
                ("ms_kernel", ctypes.c_float), ("pair_tol", ctypes.c_double)]

_lib = None


def load() -> ctypes.CDLL:
    """Loads libbarytreek_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `python -m barytreek_b200.build` "
                              "(the CUDA path has no fallback)")
        lib = ctypes.CDLL(LIB_PATH)
        for name, args in SIGNATURES.items():
            f = getattr(lib, name)
            f.argtypes = args
            f.restype = _RESTYPES.get(name, ctypes.c_int)
        _lib = lib
    return _lib


def check(status: int) -> None:
    if status != OK:
        raise BtkError(status, load().btk_last_error().decode(errors="replace"))


def ptr(a) -> int | None:
    """Address of a numpy array or torch tensor (None passes NULL)."""
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        return a.ctypes.data
    return a.data_ptr()
