"""TEST INFRASTRUCTURE ONLY — the CPU oracle for the treecode evaluation path.

Two ctypes wrappers, used only by tests/, ``__graft_entry__.smoke()`` and the
CPU-baseline leg of ``bench.py``; the product package never imports this:

* :class:`Oracle` — ``liboracle.so``, the project's serial FP64 C restatement
  of the reference's upward pass, interactions, downward pass and direct sum
  (``btk_oracle.c``; citations to the reference's files are in that source).
* :class:`RefLib` — ``_ref/libbtkref.so``, BarytreeK's own unmodified sources
  compiled against the project's Kokkos-API host shim (``Makefile``). It is
  present where the reference tree was available at build time; it pins the
  restatement and the golden fixtures, and is the timed CPU baseline.

Panel records are handled as numpy structured arrays with the reference's
byte layouts (src/structs.hpp:24-75).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

# src/structs.hpp:24-39 (TreePanel_2d, 80 bytes)
PANEL2_DTYPE = np.dtype({
    "names": ["id", "level", "parent_id", "child", "is_leaf", "max_x", "min_x", "max_y", "min_y",
              "radius", "point_count"],
    "formats": ["<i4", "<i4", "<i4", ("<i4", 4), "u1", "<f8", "<f8", "<f8", "<f8", "<f8", "<i4"],
    "offsets": [0, 4, 8, 12, 28, 32, 40, 48, 56, 64, 72],
    "itemsize": 80,
})
# src/structs.hpp:41-64 (TreePanel_3d, 112 bytes)
PANEL3_DTYPE = np.dtype({
    "names": ["id", "level", "parent_id", "child", "is_leaf", "max_x", "min_x", "max_y", "min_y",
              "min_z", "max_z", "radius", "point_count"],
    "formats": ["<i4", "<i4", "<i4", ("<i4", 8), "u1", "<f8", "<f8", "<f8", "<f8", "<f8", "<f8", "<f8",
                "<i4"],
    "offsets": [0, 4, 8, 12, 44, 48, 56, 64, 72, 80, 88, 96, 104],
    "itemsize": 112,
})
# src/structs.hpp:71-75 (interact_pair, 12 bytes)
PAIR_DTYPE = np.dtype([("target_panel", "<i4"), ("source_panel", "<i4"), ("interact_type", "<i4")])

POT, VEL, FIELD = 0, 1, 2


def ncomp(dim: int, kind: int) -> int:
    return 1 if kind == POT else (3 if kind == VEL else 1 + dim)


def _p(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def _f64(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.float64)


def build(quiet: bool = True) -> None:
    """Compile liboracle.so (and _ref/libbtkref.so when the reference tree exists)."""
    subprocess.run(["make", "-C", HERE, "all"], check=True,
                   stdout=subprocess.DEVNULL if quiet else None)


class Oracle:
    """ctypes wrapper of liboracle.so (the C restatement)."""

    def __init__(self, path: str | None = None):
        path = path or os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        self.lib = ctypes.CDLL(path)
        L = self.lib
        vp, ci, cd = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
        L.bto_interp_basis.argtypes = [vp, cd, cd, cd, ci]
        L.bto_nodes.argtypes = [vp, cd, cd, ci]
        L.bto_upward.argtypes = [ci, ci, ci, vp, vp, vp, vp, ci, vp, vp, ci, vp, vp]
        L.bto_interactions.argtypes = [ci, ci, ci, cd, ci, ci, vp, vp, vp, ci, vp, vp, vp, vp, vp, vp, vp, vp,
                                       vp, ci, vp, ci, vp, ci, vp, ci, vp, ci, vp, vp]
        L.bto_downward.argtypes = [ci, ci, ci, ci, ci, vp, vp, vp, ci, vp, vp, ci, vp, vp, vp]
        L.bto_direct.argtypes = [ci, ci, cd, ci, vp, vp, vp, ci, vp, vp, vp, vp, vp]
        L.bto_solve_degrees.argtypes = [ci, ci, ci, cd, ci, ci, vp, vp, vp, ci, vp, vp, vp, vp, vp, ci, vp, vp, ci,
                                        vp, vp, ci, vp, ci, vp, vp, ci, vp, vp, ci, vp, vp]

    def solve_degrees(self, tree, kind, q, deg_pc=None, deg_cp=None, deg_cc=None):
        """Treecode with one degree per far-field pair (bto_solve_degrees)."""
        dim, eps, thresh = tree["dim"], tree["eps"], tree["thresh"]
        tg = [_f64(a) for a in tree["targets"]] + [None] * (3 - dim)
        sc = [_f64(a) for a in tree["sources"]] + [None] * (3 - dim)
        q = _f64(q)
        nt, ns = len(tg[0]), len(sc[0])
        out = np.zeros((ncomp(dim, kind), nt))
        L = {k: np.ascontiguousarray(tree[k], PAIR_DTYPE) for k in ("pp", "pc", "cp", "cc")}
        dg = [None if d is None else np.ascontiguousarray(d, np.int32) for d in (deg_pc, deg_cp, deg_cc)]
        rc = self.lib.bto_solve_degrees(
            dim, kind, tree["degree"], eps, thresh, nt, _p(tg[0]), _p(tg[1]), _p(tg[2]), ns, _p(sc[0]), _p(sc[1]),
            _p(sc[2]), _p(q), _p(tree["panels_t"]), len(tree["panels_t"]),
            _p(np.ascontiguousarray(tree["inside_t"], np.int32)), _p(tree["panels_s"]), len(tree["panels_s"]),
            _p(np.ascontiguousarray(tree["inside_s"], np.int32)), _p(L["pp"]), len(L["pp"]), _p(L["pc"]),
            len(L["pc"]), _p(dg[0]), _p(L["cp"]), len(L["cp"]), _p(dg[1]), _p(L["cc"]), len(L["cc"]), _p(dg[2]),
            _p(out))
        if rc:
            raise RuntimeError("bto_solve_degrees failed")
        return out

    def interp_basis(self, x, lo, hi, n):
        out = np.zeros(n + 1)
        self.lib.bto_interp_basis(_p(out), x, lo, hi, n)
        return out

    def nodes(self, lo, hi, n):
        out = np.zeros(n + 1)
        self.lib.bto_nodes(_p(out), lo, hi, n)
        return out

    def direct(self, dim, kind, eps, targets, sources, q):
        t = [_f64(a) for a in targets] + [None] * (3 - len(targets))
        s = [_f64(a) for a in sources] + [None] * (3 - len(sources))
        q = _f64(q)
        nt, ns = len(t[0]), len(s[0])
        out = np.zeros((ncomp(dim, kind), nt))
        self.lib.bto_direct(dim, kind, eps, nt, _p(t[0]), _p(t[1]), _p(t[2]), ns, _p(s[0]), _p(s[1]),
                            _p(s[2]), _p(q), _p(out))
        return out

    def solve(self, tree, kind, q, targets=None, sources=None):
        """Full upward -> interactions -> downward on a tree description.

        ``tree`` is a dict with dim, degree, eps, thresh, panels_t, panels_s,
        level_start_t/_s, leaf_of_s, inside_t/_s and the four pair lists, plus
        ``targets``/``sources`` coordinate tuples. Returns dict(psw, ptw_mid,
        mid, out) mirroring RefLib.solve.
        """
        dim, deg, eps, thresh = tree["dim"], tree["degree"], tree["eps"], tree["thresh"]
        tg = [_f64(a) for a in tree["targets"]] + [None] * (3 - dim)
        sc = [_f64(a) for a in tree["sources"]] + [None] * (3 - dim)
        q = _f64(q)
        nt, ns = len(tg[0]), len(sc[0])
        ipc = (deg + 1) ** dim
        nc = ncomp(dim, kind)
        Pt, Ps = len(tree["panels_t"]), len(tree["panels_s"])
        psw = np.zeros((Ps, ipc))
        ls_s = np.ascontiguousarray(tree["level_start_s"], np.int32)
        ls_t = np.ascontiguousarray(tree["level_start_t"], np.int32)
        self.lib.bto_upward(dim, deg, ns, _p(sc[0]), _p(sc[1]), _p(sc[2]), _p(q), Ps,
                            _p(tree["panels_s"]), _p(ls_s), len(ls_s) - 1,
                            _p(np.ascontiguousarray(tree["leaf_of_s"], np.int32)), _p(psw))
        ptw = np.zeros((nc, Pt, ipc))
        out = np.zeros((nc, nt))
        L = {k: np.ascontiguousarray(tree[k], PAIR_DTYPE) for k in ("pp", "pc", "cp", "cc")}
        self.lib.bto_interactions(dim, kind, deg, eps, thresh, nt, _p(tg[0]), _p(tg[1]), _p(tg[2]), ns,
                                  _p(sc[0]), _p(sc[1]), _p(sc[2]), _p(q), _p(tree["panels_t"]),
                                  _p(np.ascontiguousarray(tree["inside_t"], np.int32)), _p(tree["panels_s"]),
                                  _p(np.ascontiguousarray(tree["inside_s"], np.int32)),
                                  _p(L["pp"]), len(L["pp"]), _p(L["pc"]), len(L["pc"]), _p(L["cp"]),
                                  len(L["cp"]), _p(L["cc"]), len(L["cc"]), _p(psw), Pt, _p(ptw), _p(out))
        mid, ptw_mid = out.copy(), ptw.copy()
        self.lib.bto_downward(dim, nc, deg, thresh, nt, _p(tg[0]), _p(tg[1]), _p(tg[2]), Pt,
                              _p(tree["panels_t"]), _p(ls_t), len(ls_t) - 1,
                              _p(np.ascontiguousarray(tree["inside_t"], np.int32)), _p(ptw), _p(out))
        return {"psw": psw, "ptw_mid": ptw_mid, "mid": mid, "out": out}


class RefLib:
    """ctypes wrapper of _ref/libbtkref.so (the reference compiled against the shim)."""

    PATH = os.path.join(HERE, "_ref", "libbtkref.so")

    @classmethod
    def available(cls) -> bool:
        return os.path.exists(cls.PATH)

    def __init__(self, threads: int = 1):
        if not self.available():
            raise FileNotFoundError(self.PATH)
        self.lib = ctypes.CDLL(self.PATH)
        L = self.lib
        vp, ci, cd = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
        L.btkref_create.restype = vp
        L.btkref_create.argtypes = [ci, ci, vp, vp, vp, ci, vp, vp, vp, ci, ci, cd, cd]
        L.btkref_destroy.argtypes = [vp]
        L.btkref_info.argtypes = [vp, vp]
        L.btkref_get_config.argtypes = [vp, vp]
        L.btkref_get_tree.argtypes = [vp, ci, vp, vp, vp, vp]
        L.btkref_get_lists.argtypes = [vp, vp, vp, vp, vp, vp]
        L.btkref_solve.argtypes = [vp, ci, ci, vp, vp, vp, vp, vp]
        L.btkref_direct.argtypes = [ci, ci, ci, vp, vp, vp, ci, vp, vp, vp, vp, cd, vp]
        L.btkref_time_sample_3d.argtypes = [vp, ci, ci, vp, vp, vp, vp]
        L.btkref_solve_leaves.argtypes = [vp, ci, vp, ci, vp, vp]
        L.btkref_read_namelist.argtypes = [ctypes.c_char_p, ci, vp]
        L.btkref_set_threads.argtypes = [ci]
        self.set_threads(threads)

    def set_threads(self, n: int) -> None:
        self.lib.btkref_set_threads(n)

    def max_threads(self) -> int:
        return self.lib.btkref_max_threads()

    def sizeof(self, which: int) -> int:
        return self.lib.btkref_sizeof(which)

    def read_namelist(self, path: str, dim: int) -> bytes:
        buf = ctypes.create_string_buffer(64)
        rc = self.lib.btkref_read_namelist(path.encode(), dim, buf)
        if rc:
            raise RuntimeError("namelist not found")
        return buf.raw

    def create(self, dim, targets, sources=None, degree=8, cluster_size=100, theta=0.7, eps=1e-4):
        return RefTree(self, dim, targets, sources, degree, cluster_size, theta, eps)

    def direct(self, dim, kind, eps, targets, sources, q):
        t = [_f64(a) for a in targets] + [None] * (3 - len(targets))
        s = [_f64(a) for a in sources] + [None] * (3 - len(sources))
        q = _f64(q)
        nt, ns = len(t[0]), len(s[0])
        out = np.zeros((3 if kind == VEL else 1, nt))
        self.lib.btkref_direct(dim, kind, nt, _p(t[0]), _p(t[1]), _p(t[2]), ns, _p(s[0]), _p(s[1]), _p(s[2]),
                               _p(q), eps, _p(out))
        return out


class RefTree:
    """One reference tree + interaction lists (targets = sources unless split)."""

    def __init__(self, ref, dim, targets, sources, degree, cluster_size, theta, eps):
        self.ref, self.dim, self.eps = ref, dim, eps
        self.targets = tuple(_f64(a) for a in targets)
        self.split = sources is not None
        self.sources = tuple(_f64(a) for a in sources) if self.split else self.targets
        t = list(self.targets) + [None] * (3 - dim)
        s = list(self.sources) + [None] * (3 - dim) if self.split else [None, None, None]
        self.h = ctypes.c_void_p(ref.lib.btkref_create(dim, len(t[0]), _p(t[0]), _p(t[1]), _p(t[2]),
                                                       len(self.sources[0]), _p(s[0]), _p(s[1]), _p(s[2]),
                                                       degree, cluster_size, theta, eps))
        info = np.zeros(13, np.int32)
        ref.lib.btkref_info(self.h, _p(info))
        self.info = info
        cfg = ctypes.create_string_buffer(64)
        ref.lib.btkref_get_config(self.h, cfg)
        self.config_bytes = cfg.raw
        self.degree, self.thresh, self.ipc = int(info[12]), int(info[11]), int(info[10])
        dt = PANEL2_DTYPE if dim == 2 else PANEL3_DTYPE
        self.trees = []
        for which, (P, levels, n) in enumerate([(info[1], info[2], len(self.targets[0])),
                                                (info[3], info[4], len(self.sources[0]))]):
            panels = np.zeros(P, dt)
            ls = np.zeros(levels + 1, np.int32)
            leaf = np.zeros(n, np.int32)
            inside = np.zeros((P, self.thresh), np.int32)
            ref.lib.btkref_get_tree(self.h, which, _p(panels), _p(ls), _p(leaf), _p(inside))
            self.trees.append({"panels": panels, "level_start": ls, "leaf_of": leaf, "inside": inside})
        self.all = np.zeros(info[9], PAIR_DTYPE)
        self.lists = {k: np.zeros(info[5 + i], PAIR_DTYPE) for i, k in enumerate(("pp", "pc", "cp", "cc"))}
        ref.lib.btkref_get_lists(self.h, _p(self.all), *[_p(self.lists[k]) for k in ("pp", "pc", "cp", "cc")])

    def __del__(self):
        try:
            self.ref.lib.btkref_destroy(self.h)
        except Exception:
            pass

    def as_dict(self):
        """Tree description accepted by Oracle.solve."""
        t, s = self.trees[0], self.trees[1]
        return {"dim": self.dim, "degree": self.degree, "eps": self.eps, "thresh": self.thresh,
                "targets": self.targets, "sources": self.sources,
                "panels_t": t["panels"], "panels_s": s["panels"],
                "level_start_t": t["level_start"], "level_start_s": s["level_start"],
                "leaf_of_s": s["leaf_of"], "inside_t": t["inside"], "inside_s": s["inside"], **self.lists}

    def solve(self, kind, q, fixed=True):
        nt = len(self.targets[0])
        nc = 3 if kind == VEL else 1
        Pt, Ps = int(self.info[1]), int(self.info[3])
        psw = np.zeros((Ps, self.ipc))
        ptw = np.zeros((nc, Pt, self.ipc))
        mid = np.zeros((nc, nt))
        out = np.zeros((nc, nt))
        rc = self.ref.lib.btkref_solve(self.h, kind, int(fixed), _p(_f64(q)), _p(psw), _p(ptw), _p(mid), _p(out))
        if rc:
            raise RuntimeError(f"btkref_solve rc={rc}")
        return {"psw": psw, "ptw_mid": ptw, "mid": mid, "out": out}

    def solve_leaves(self, kind, q, leaves):
        """The fixed solve at the targets of the given leaf panels only (upward
        pass in full, interaction pairs whose target is one of those leaves or
        an ancestor, downward pass along those panels). Returns (ncomp, nt);
        only the sampled leaves' targets hold the full solution."""
        nt = len(self.targets[0])
        nc = 3 if kind == VEL else 1
        leaves = np.ascontiguousarray(leaves, dtype=np.int32)
        out = np.zeros((nc, nt))
        rc = self.ref.lib.btkref_solve_leaves(self.h, kind, _p(_f64(q)), len(leaves), _p(leaves), _p(out))
        if rc:
            raise RuntimeError(f"btkref_solve_leaves rc={rc}")
        return out

    def leaf_targets(self, leaves):
        """Original indices of the targets in the given leaf panels."""
        t = self.trees[0]
        cnt = t["panels"]["point_count"]
        return np.concatenate([t["inside"][L, :cnt[L]] for L in leaves]).astype(np.int64)

    def time_sample_3d(self, kind, stride, q):
        sec, scale, ev = np.zeros(8), np.zeros(8), np.zeros(2)
        rc = self.ref.lib.btkref_time_sample_3d(self.h, kind, stride, _p(_f64(q)), _p(sec), _p(scale), _p(ev))
        if rc:
            raise RuntimeError(f"btkref_time_sample_3d rc={rc}")
        return sec, scale, ev

    def leaves_on_last_level_only(self) -> bool:
        t = self.trees[0]
        p = t["panels"]
        last = len(t["level_start"]) - 2
        return bool(np.all(p["level"][p["is_leaf"] == 1] == last))
