"""Host-side mirror of the reference's treecode interface, over the C ABI.

Functions named after the reference's host calls (``read_run_config``,
``tree_construction``, ``dual_tree_traversal``, ``split_interactions``) return
numpy arrays in the reference's layouts; :class:`Treecode` runs the
reference's phase sequence (examples/example_poisson_3d.cpp:72-156: tree,
traversal, split, upward pass, interactions, downward pass) on the GPU through
a resident plan.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from ._lib import (KIND_FIELD, KIND_POT, KIND_VEL, PAIR_DTYPE, PANEL2_DTYPE, PANEL3_DTYPE, PREC_FP64, PREC_MIXED,
                   RunConfig, TreeInfo, check, load, ptr)

__all__ = ["make_run_config", "read_run_config", "tree_construction", "dual_tree_traversal", "split_interactions",
           "cc_operator_groups",
           "HostTree", "Treecode", "ncomp", "KIND_POT", "KIND_VEL", "KIND_FIELD", "PREC_FP64", "PREC_MIXED"]


def ncomp(dim: int, kind: int) -> int:
    return 1 if kind == KIND_POT else (3 if kind == KIND_VEL else 1 + dim)


def make_run_config(dim: int, degree: int = 8, cluster_size: int = 100, theta: float = 0.7,
                    eps: float = 1e-4) -> RunConfig:
    """RunConfig with the fields read_run_config would set (src/read_namelist.cpp:24-38),
    except that degrees up to the device limit (12) are kept instead of clamped to 10."""
    cfg = RunConfig()
    cfg.dim = dim
    cfg.interp_degree = degree
    cfg.interp_point_count = (degree + 1) ** dim
    cfg.fmm_cluster_thresh = cluster_size if cluster_size > 0 else (2 ** dim) * cfg.interp_point_count
    cfg.fmm_theta = theta
    cfg.ker_eps = eps
    cfg.mpi_p, cfg.mpi_id = 1, 0
    return cfg


def read_run_config(path: str, dim: int) -> RunConfig:
    """src/read_namelist.cpp:10-43 (``dim`` preset, as the reference drivers do)."""
    cfg = RunConfig()
    cfg.dim = dim
    cfg.fmm_theta = 0.7
    cfg.ker_eps = -1.0
    check(load().btk_read_run_config(path.encode(), ctypes.byref(cfg)))
    return cfg


class HostTree:
    """Output of tree_construction: reference layouts as numpy arrays.

    panels (PANEL2_DTYPE / PANEL3_DTYPE records), level_start int32[levels+1],
    point_leaf_panel int32[n], panel_points_inside int32[panel_count, thresh].
    A tree built on the device carries its leaf rows as ``leaf_order`` (the
    rows concatenated) and forms panel_points_inside only when asked.
    """

    def __init__(self, dim, panels, level_start, point_leaf_panel, panel_points_inside=None, leaf_order=None,
                 thresh=None):
        self.dim = dim
        self.panels = panels
        self.level_start = level_start
        self.point_leaf_panel = point_leaf_panel
        self._inside = panel_points_inside
        self.leaf_order = leaf_order
        self.thresh = thresh if thresh is not None else (panel_points_inside.shape[1] if panel_points_inside is not None
                                                         else 0)

    @property
    def has_inside(self) -> bool:
        return self._inside is not None

    @property
    def panel_points_inside(self) -> np.ndarray:
        if self._inside is None:
            inside = np.zeros((len(self.panels), self.thresh), np.int32)
            off = 0
            for i in np.flatnonzero(self.panels["is_leaf"] != 0):
                c = int(self.panels["point_count"][i])
                inside[i, :c] = self.leaf_order[off:off + c]
                off += c
            self._inside = inside
        return self._inside

    @property
    def panel_count(self) -> int:
        return len(self.panels)

    @property
    def levels(self) -> int:
        return len(self.level_start) - 1

    def tree_info(self) -> TreeInfo:
        ti = TreeInfo()
        ti.panel_count = self.panel_count
        ti.levels = self.levels
        ti.level_start = self.level_start.ctypes.data_as(ctypes.POINTER(ctypes.c_int))
        return ti


def _copy_out(addr: int, dtype, count: int) -> np.ndarray:
    out = np.empty(count, dtype)
    if count:
        ctypes.memmove(out.ctypes.data, addr, out.nbytes)
    return out


def tree_construction_device(cfg: RunConfig, coords, stream=None) -> HostTree:
    """The same tree from CUDA-tensor coordinates (btk_tree_construction_*_device):
    point work on the GPU; panels and leaf rows returned to the host."""
    import torch
    L = load()
    dim = cfg.dim
    n = int(coords[0].numel())
    dev = coords[0].device
    leaf_of = torch.empty(max(n, 1), dtype=torch.int32, device=dev)
    order = torch.empty(max(n, 1), dtype=torch.int32, device=dev)
    info = TreeInfo()
    panels_p = ctypes.c_void_p()
    st = stream if stream is not None else torch.cuda.current_stream(dev).cuda_stream
    if dim == 2:
        check(L.btk_tree_construction_2d_device(ctypes.byref(cfg), ctypes.byref(info), ptr(coords[0]), ptr(coords[1]),
                                                n, ctypes.byref(panels_p), ptr(leaf_of), ptr(order), st))
    else:
        check(L.btk_tree_construction_3d_device(ctypes.byref(cfg), ctypes.byref(info), ptr(coords[0]), ptr(coords[1]),
                                                ptr(coords[2]), n, ctypes.byref(panels_p), ptr(leaf_of), ptr(order),
                                                st))
    try:
        panels = _copy_out(panels_p.value, PANEL2_DTYPE if dim == 2 else PANEL3_DTYPE, info.panel_count)
        ls = _copy_out(ctypes.cast(info.level_start, ctypes.c_void_p).value, np.int32, info.levels + 1)
    finally:
        L.btk_free(panels_p)
        L.btk_free(ctypes.cast(info.level_start, ctypes.c_void_p))
    return HostTree(dim, panels, ls, leaf_of[:n].cpu().numpy(), leaf_order=order[:n].cpu().numpy(),
                    thresh=cfg.fmm_cluster_thresh)


def tree_construction(cfg: RunConfig, coords) -> HostTree:
    """blfmm_tree_construction_2d/3d (src/tree_construction.cpp), bit-identical."""
    L = load()
    dim = cfg.dim
    xyz = [np.ascontiguousarray(c, np.float64) for c in coords]
    n = len(xyz[0])
    info = TreeInfo()
    panels_p = ctypes.c_void_p()
    inside_p = ctypes.c_void_p()
    leaf = np.zeros(n, np.int32)
    if dim == 2:
        check(L.btk_tree_construction_2d(ctypes.byref(cfg), ctypes.byref(info), ptr(xyz[0]), ptr(xyz[1]), n,
                                         ctypes.byref(panels_p), ptr(leaf), ctypes.byref(inside_p)))
    else:
        check(L.btk_tree_construction_3d(ctypes.byref(cfg), ctypes.byref(info), ptr(xyz[0]), ptr(xyz[1]),
                                         ptr(xyz[2]), n, ctypes.byref(panels_p), ptr(leaf), ctypes.byref(inside_p)))
    P = info.panel_count
    try:
        panels = _copy_out(panels_p.value, PANEL2_DTYPE if dim == 2 else PANEL3_DTYPE, P)
        inside = _copy_out(inside_p.value, np.int32, P * cfg.fmm_cluster_thresh).reshape(P, cfg.fmm_cluster_thresh)
        ls = _copy_out(ctypes.cast(info.level_start, ctypes.c_void_p).value, np.int32, info.levels + 1)
    finally:
        L.btk_free(panels_p)
        L.btk_free(inside_p)
        L.btk_free(ctypes.cast(info.level_start, ctypes.c_void_p))
    return HostTree(dim, panels, ls, leaf, inside)


def dual_tree_traversal(cfg: RunConfig, target: HostTree, source: HostTree | None = None) -> np.ndarray:
    """dual_tree_traversal_2d/3d (src/interaction_list.cpp); updates cfg's counts."""
    L = load()
    source = source or target
    out = ctypes.c_void_p()
    fn = L.btk_dual_tree_traversal_2d if cfg.dim == 2 else L.btk_dual_tree_traversal_3d
    check(fn(ctypes.byref(cfg), ptr(target.panels), ptr(source.panels), ctypes.byref(out)))
    try:
        return _copy_out(out.value, PAIR_DTYPE, cfg.fmm_interaction_count)
    finally:
        L.btk_free(out)


def dual_tree_traversal_device(cfg: RunConfig, target: HostTree, source: HostTree | None = None,
                               stream=None) -> np.ndarray:
    """The same list as dual_tree_traversal, computed on the GPU
    (btk_dual_tree_traversal_*_device); updates cfg's counts."""
    import torch
    L = load()
    source = source or target
    out = ctypes.c_void_p()
    fn = L.btk_dual_tree_traversal_2d_device if cfg.dim == 2 else L.btk_dual_tree_traversal_3d_device
    st = stream if stream is not None else torch.cuda.current_stream().cuda_stream
    check(fn(ctypes.byref(cfg), ptr(target.panels), target.panel_count, ptr(source.panels), source.panel_count,
             ctypes.byref(out), st))
    try:
        return _copy_out(out.value, PAIR_DTYPE, cfg.fmm_interaction_count)
    finally:
        L.btk_free(out)


def split_interactions(cfg: RunConfig, interactions: np.ndarray):
    """split_interactions (src/interaction_list.cpp:252-277) -> (pp, pc, cp, cc)."""
    lists = [np.zeros(c, PAIR_DTYPE) for c in (cfg.fmm_pp_count, cfg.fmm_pc_count, cfg.fmm_cp_count,
                                               cfg.fmm_cc_count)]
    check(load().btk_split_interactions(ptr(interactions), len(interactions), *[ptr(l) for l in lists]))
    return tuple(lists)


def cc_operator_groups(dim: int, target: HostTree, cc_list: np.ndarray, source: HostTree | None = None):
    """Group id of every CC pair under the shared-matrix CC form (host only):
    pairs with equal target level, source level and lattice offset share one.
    Returns (group_of_pair int32[n_cc], n_groups); n_groups is 0 (ids -1) when
    the trees are not midpoint subdivisions of one common root box."""
    g = np.full(len(cc_list), -1, np.int32)
    n = ctypes.c_int(0)
    src = source.panels if source is not None else None
    check(load().btk_cc_operator_groups(dim, ptr(target.panels), target.panel_count, ptr(src) if src is not None else None,
                                        source.panel_count if source is not None else 0,
                                        ptr(cc_list) if len(cc_list) else None, len(cc_list),
                                        ptr(g) if len(g) else None, ctypes.byref(n)))
    return g, n.value


class Treecode:
    """A resident treecode plan: targets = sources unless ``sources`` is given.

    ``coords``: tuple of dim float64 arrays (host). Trees and lists are built
    with the bit-identical host functions (``device_tree=True``: the same tree
    and lists built on the GPU from the device copies of the points), then a device plan holds the
    leaf ordering, geometry and interaction work lists. ``cc_operators=True`` applies the CC pairs of
    a fixed-degree plan as shared kernel matrices (pairs grouped by level and lattice offset).
    ``leaf_far_pairs=True`` (per-pair plans) lets the learned degree choice approximate well-separated
    PP pairs as target points x source-leaf proxies, with the direct evaluation as an option.
    ``tile_targets=128`` runs the interaction kernels on tiles of 128 targets (64-thread blocks) instead of 256.
    :meth:`solve` takes
    charges (numpy or a CUDA tensor) and returns a CUDA tensor
    ``[ncomp, n_targets]`` in the original point order.
    """

    def __init__(self, coords, sources=None, *, degree=8, cluster_size=100, theta=0.7, eps=1e-4, kind=KIND_POT,
                 precision=PREC_FP64, degree_mode=_lib.DEGREE_FIXED, degree_min=1, work_split=0, device_tree=False,
                 cc_operators=False, leaf_far_pairs=False, leaf_far_theta=0.0, tile_targets=0, device="cuda"):
        import torch

        self.dim = len(coords)
        self.kind, self.precision = kind, precision
        self.degree_mode, self.degree_min = degree_mode, degree_min
        self.work_split = work_split
        self.cc_operators = bool(cc_operators)
        self.leaf_far_pairs = bool(leaf_far_pairs)
        self.leaf_far_theta = float(leaf_far_theta)
        self.tile_targets = int(tile_targets)
        self.ncomp = ncomp(self.dim, kind)
        self.cfg = make_run_config(self.dim, degree, cluster_size, theta, eps)
        self.targets = tuple(np.ascontiguousarray(c, np.float64) for c in coords)
        self.sources = tuple(np.ascontiguousarray(c, np.float64) for c in sources) if sources is not None else None
        self.device = torch.device(device)
        dev = self.device
        self._t = [torch.from_numpy(c).to(dev) for c in self.targets]
        # device_tree: the same tree built from the device copies of the points
        self.tree_t = (tree_construction_device(self.cfg, self._t) if device_tree
                       else tree_construction(self.cfg, self.targets))
        self.tree_s = tree_construction(self.cfg, self.sources) if self.sources is not None else None
        self.interactions = (dual_tree_traversal_device(self.cfg, self.tree_t, self.tree_s) if device_tree
                             else dual_tree_traversal(self.cfg, self.tree_t, self.tree_s))
        self.lists = split_interactions(self.cfg, self.interactions)
        self.nt = len(self.targets[0])
        self.ns = len(self.sources[0]) if self.sources is not None else self.nt
        self._s = [torch.from_numpy(c).to(dev) for c in self.sources] if self.sources is not None else self._t
        self._plan = ctypes.c_void_p()
        self._create_plan()

    def _create_plan(self):
        import torch

        d = _lib.PlanDesc()
        d.cfg = self.cfg
        d.point_count_target, d.point_count_source = self.nt, self.ns
        self._ti_t = self.tree_t.tree_info()
        d.tree_target = ctypes.pointer(self._ti_t)
        d.panels_target = ptr(self.tree_t.panels)
        # a device-built tree hands over its leaf order through point_leaf_panel (one tree)
        d.panel_points_inside_target = (ptr(self.tree_t.panel_points_inside)
                                        if self.tree_t.has_inside or self.tree_s is not None else None)
        src = self.tree_s or self.tree_t
        if self.tree_s is not None:
            self._ti_s = self.tree_s.tree_info()
            d.tree_source = ctypes.pointer(self._ti_s)
            d.panels_source = ptr(self.tree_s.panels)
            d.panel_points_inside_source = ptr(self.tree_s.panel_points_inside)
        d.point_leaf_panel_source = ptr(src.point_leaf_panel)
        d.pp_list, d.pc_list, d.cp_list, d.cc_list = [ptr(l) if len(l) else None for l in self.lists]
        d.kind, d.precision = self.kind, self.precision
        d.degree_mode, d.degree_min = self.degree_mode, self.degree_min
        d.work_split = self.work_split
        d.cc_operators = int(self.cc_operators)
        d.leaf_far_pairs = int(self.leaf_far_pairs)
        d.leaf_far_theta = self.leaf_far_theta
        d.tile_targets = self.tile_targets
        stream = torch.cuda.current_stream(self.device).cuda_stream
        check(load().btk_plan_create(ctypes.byref(self._plan), ctypes.byref(d), stream))

    def set_degree_rule(self, rule: int):
        """_lib.DEGREE_RULE_THRESHOLD or _lib.DEGREE_RULE_COST for learned solves."""
        check(load().btk_plan_set_degree_rule(self._plan, rule))

    def set_degrees(self, deg_pc=None, deg_cp=None, deg_cc=None):
        """Per-pair degrees for a degree_mode=DEGREE_PER_PAIR plan (host arrays in list order)."""
        arrs = [None if d is None else np.ascontiguousarray(d, np.int32) for d in (deg_pc, deg_cp, deg_cc)]
        check(load().btk_plan_set_degrees(self._plan, *[ptr(a) for a in arrs]))

    def stats(self) -> dict:
        s = _lib.PlanStats()
        check(load().btk_plan_stats_get(self._plan, ctypes.byref(s)))
        return {k: getattr(s, k) for k, _ in s._fields_}

    def evals(self) -> int:
        s = self.stats()
        return s["evals_pp"] + s["evals_pc"] + s["evals_cp"] + s["evals_cc"]

    def solve(self, charges, out=None):
        import torch

        q = charges if isinstance(charges, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(charges, np.float64))
        q = q.to(self.device, torch.float64).contiguous()
        if out is None:
            out = torch.empty((self.ncomp, self.nt), dtype=torch.float64, device=self.device)
        t, s = self._t, self._s
        stream = torch.cuda.current_stream(self.device).cuda_stream
        z_t = ptr(t[2]) if self.dim == 3 else None
        z_s = ptr(s[2]) if self.dim == 3 else None
        check(load().btk_plan_execute(self._plan, ptr(t[0]), ptr(t[1]), z_t, ptr(s[0]), ptr(s[1]), z_s, ptr(q),
                                      ptr(out), stream))
        return out

    def solve_learned(self, charges, selector, tol=1e-6, pair_tol=None, degree_lo=4, out=None):
        """Learned-degree solve with a 1% FP64 direct-sum audit and fallback
        (btk_plan_execute_learned). Returns (out tensor, report dict)."""
        import torch

        q = charges if isinstance(charges, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(charges, np.float64))
        q = q.to(self.device, torch.float64).contiguous()
        if out is None:
            out = torch.empty((self.ncomp, self.nt), dtype=torch.float64, device=self.device)
        pair_tol = 0.0 if pair_tol is None else pair_tol  # 0: the plan's adaptive per-pair tolerance
        t, s = self._t, self._s
        stream = torch.cuda.current_stream(self.device).cuda_stream
        z_t = ptr(t[2]) if self.dim == 3 else None
        z_s = ptr(s[2]) if self.dim == 3 else None
        rep = _lib.LearnedReport()
        check(load().btk_plan_execute_learned(self._plan, selector.handle(), tol, pair_tol, degree_lo, ptr(t[0]),
                                              ptr(t[1]), z_t, ptr(s[0]), ptr(s[1]), z_s, ptr(q), ptr(out),
                                              ctypes.byref(rep), stream))
        r = {k: getattr(rep, k) for k, _ in rep._fields_ if k != "degree_hist"}
        r["degree_hist"] = list(rep.degree_hist)
        return out, r

    def set_wait_limit(self, polls: int):
        """Polls of each chunk barrier before the interaction kernel gives up
        (btk_plan_set_wait_limit); 0 gives up at once, < 0 restores the default."""
        check(load().btk_plan_set_wait_limit(self._plan, int(polls)))

    def audit_targets(self) -> np.ndarray:
        """Original indices of the targets the learned solve's audit checks."""
        n = ctypes.c_int(0)
        check(load().btk_plan_audit_targets(self._plan, ctypes.byref(n), None))
        out = np.zeros(n.value, np.int32)
        if n.value:
            check(load().btk_plan_audit_targets(self._plan, ctypes.byref(n), ptr(out)))
        return out

    def last_timing(self) -> dict:
        ms = (ctypes.c_float * 5)()
        check(load().btk_plan_last_timing(self._plan, ms))
        return {"upward": ms[0], "interactions": ms[1], "downward": ms[2], "total": ms[3],
                "interaction_kernel": ms[4]}

    def close(self):
        if self._plan:
            load().btk_plan_destroy(self._plan)
            self._plan = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
