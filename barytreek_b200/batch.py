"""Batches of independent problems in one forest plan, and the leaf-size /
work-split autotuner.

:class:`Batch` wraps btk_batch_*: every problem's tree and lists come from the
host tree functions with that problem's own leaf size, the trees are merged
into one level-major forest, and each solve is one CUDA graph (gathers, upward
pass, ONE persistent interaction launch over all problems, downward pass).

:class:`Autotuner` picks, per size bucket (problems with 2^k <= N < 2^(k+1)),
the leaf size and the work split (work items per persistent-grid slot, the
tile granularity of the scheduler) that give the shortest batched solve. It
times mini-batches of representative problems of the bucket drawn from the
same generator as the workload, so the choice reflects throughput inside a
batch, not the latency of one small problem alone.
"""
from __future__ import annotations

import ctypes
import json
import math
import os
import time

import numpy as np

from . import _lib, datagen
from ._lib import KIND_POT, PREC_MIXED, check, load, ptr

__all__ = ["Batch", "Autotuner", "bucket_of", "cfg3_problems"]

DEFAULT_TABLE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "autotune_table.json")


def bucket_of(n: int) -> int:
    """Size bucket: floor(log2 N), with N = 2^18 folded into bucket 17."""
    return min(17, max(12, int(math.floor(math.log2(max(n, 1))))))


def cfg3_problems(seed: int, count: int = 256, n_lo: int = 4096, n_hi: int = 262144):
    """Problem sizes log-uniform in [n_lo, n_hi] and Gaussian-mixture points
    with standard-normal charges (one seeded stream per problem)."""
    u = datagen.uniform(seed, 70, count)
    sizes = np.exp(np.log(n_lo) + u * (np.log(n_hi) - np.log(n_lo))).astype(np.int64)
    sizes = np.clip(sizes, n_lo, n_hi)
    return [datagen.gaussian_mixture(seed * 1000 + 17 + b, int(n)) for b, n in enumerate(sizes)]


class Batch:
    """Many independent problems (targets = sources each) solved as one plan.

    problems: list of (coords tuple, ...) where coords is a tuple of dim
    float64 arrays. cluster_size: one leaf size for all, a per-problem list, or
    None to take it from ``table`` (an :class:`Autotuner` table) by size bucket.
    """

    def __init__(self, coords_list, *, degree=6, theta=0.6, eps=1e-4, kind=KIND_POT, precision=PREC_MIXED,
                 cluster_size=None, table=None, work_split=None, tile_targets=None, device="cuda"):
        import torch

        self.dim = len(coords_list[0])
        self.sizes = np.array([len(c[0]) for c in coords_list], np.int64)
        self.offsets = np.zeros(len(coords_list) + 1, np.int32)
        self.offsets[1:] = np.cumsum(self.sizes)
        self.n = int(self.offsets[-1])
        if cluster_size is None:
            table = table or Autotuner.load()
            cluster_size = [table.leaf_for(int(n)) for n in self.sizes]
            if work_split is None:
                work_split = table.split_for_batch(self.sizes)
            if tile_targets is None:
                tile_targets = table.tile_for_batch(self.sizes)
        if np.isscalar(cluster_size):
            cluster_size = [int(cluster_size)] * len(coords_list)
        self.cluster_size = np.ascontiguousarray(cluster_size, np.int32)
        self.work_split = int(work_split or 0)
        self.tile_targets = int(tile_targets or 0)
        self.kind, self.precision = kind, precision
        self.ncomp = 1 if kind == KIND_POT else (3 if kind == _lib.KIND_VEL else 1 + self.dim)
        xyz = [np.ascontiguousarray(np.concatenate([c[d] for c in coords_list]), np.float64) for d in range(self.dim)]
        d = _lib.BatchDesc()
        d.forest.dim, d.forest.degree, d.forest.theta, d.forest.eps = self.dim, degree, theta, eps
        d.forest.n_problems = len(coords_list)
        d.forest.point_offset = ptr(self.offsets)
        d.forest.cluster_size = ptr(self.cluster_size)
        d.kind, d.precision, d.work_split = kind, precision, self.work_split
        d.tile_targets = self.tile_targets
        self.device = torch.device(device)
        self._h = ctypes.c_void_p()
        stream = torch.cuda.current_stream(self.device).cuda_stream
        t0 = time.perf_counter()
        check(load().btk_batch_create(ctypes.byref(self._h), ctypes.byref(d), ptr(xyz[0]), ptr(xyz[1]),
                                      ptr(xyz[2]) if self.dim == 3 else None, stream))
        self.setup_s = time.perf_counter() - t0

    def solve(self, charges, out=None):
        """charges: concatenated (numpy or CUDA tensor). Returns CUDA [ncomp, N]."""
        import torch

        q = charges if isinstance(charges, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(charges, np.float64))
        q = q.to(self.device, torch.float64).contiguous()
        if out is None:
            out = torch.empty((self.ncomp, self.n), dtype=torch.float64, device=self.device)
        stream = torch.cuda.current_stream(self.device).cuda_stream
        check(load().btk_batch_execute(self._h, ptr(q), ptr(out), stream))
        return out

    def split(self, out):
        """Per-problem views of a batch result."""
        return [out[:, self.offsets[b]:self.offsets[b + 1]] for b in range(len(self.sizes))]

    def stats(self) -> dict:
        s = _lib.BatchStats()
        check(load().btk_batch_stats_get(self._h, ctypes.byref(s)))
        return {k: getattr(s, k) for k, _ in s._fields_}

    def evals(self) -> int:
        s = self.stats()
        return s["evals_pp"] + s["evals_pc"] + s["evals_cp"] + s["evals_cc"]

    def close(self):
        if self._h:
            load().btk_batch_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Autotuner:
    """Per-bucket leaf size, work split and tile size (targets per work item),
    chosen by timing batched solves."""

    LEAVES = (128, 256, 512, 1024, 2048, 4096)
    SPLITS = (4, 8, 16)
    TILES = (256, 128)

    def __init__(self, table: dict | None = None, meta: dict | None = None):
        # bucket -> (leaf, split[, tile]); tables without a tile mean 256
        self.table = {int(k): tuple(v) for k, v in (table or {}).items()}
        self.meta = meta or {}

    # -- persistence
    @classmethod
    def load(cls, path: str = DEFAULT_TABLE) -> "Autotuner":
        with open(path) as f:
            z = json.load(f)
        return cls(z["table"], z.get("meta"))

    def save(self, path: str = DEFAULT_TABLE) -> None:
        with open(path, "w") as f:
            json.dump({"table": {str(k): list(v) for k, v in sorted(self.table.items())}, "meta": self.meta}, f,
                      indent=1)

    # -- lookup
    def leaf_for(self, n: int) -> int:
        b = bucket_of(n)
        if b in self.table:
            return self.table[b][0]
        near = min(self.table, key=lambda k: abs(k - b))
        return self.table[near][0]

    def _main_bucket(self, sizes) -> int:
        w = {}
        for n in sizes:
            b = bucket_of(int(n))
            w[b] = w.get(b, 0) + int(n)
        return max(w, key=w.get)

    def split_for_batch(self, sizes) -> int:
        """The work split of the bucket holding most of the batch's points."""
        return self.table.get(self._main_bucket(sizes), (0, 8))[1]

    def tile_for_batch(self, sizes) -> int:
        """The tile size of the bucket holding most of the batch's points."""
        e = self.table.get(self._main_bucket(sizes), (0, 8))
        return e[2] if len(e) > 2 else 256

    # -- tuning
    @staticmethod
    def _time_batch(coords, q, leaf, split, degree, theta, eps, kind, precision, reps, tile=256):
        import torch

        b = Batch(coords, degree=degree, theta=theta, eps=eps, kind=kind, precision=precision, cluster_size=leaf,
                  work_split=split, tile_targets=tile)
        qd = torch.from_numpy(q).cuda()
        out = torch.empty((b.ncomp, b.n), dtype=torch.float64, device="cuda")
        b.solve(qd, out)  # capture
        b.solve(qd, out)
        ts = []
        for _ in range(reps):
            b.solve(qd, out)
            ts.append(b.stats()["last_ms"])
        b.close()
        return float(np.median(ts))

    def tune(self, buckets=range(12, 18), *, points_per_batch=1 << 20, degree=6, theta=0.6, eps=1e-4,
             kind=KIND_POT, precision=PREC_MIXED, leaves=None, splits=None, tiles=None, reps=3, seed=900,
             log=None):
        """Times every leaf size (at split 8, tile 256), then every split at
        the best leaf, then every tile size at the best pair, on a mini-batch
        of representative problems per bucket."""
        leaves = tuple(leaves or self.LEAVES)
        splits = tuple(splits or self.SPLITS)
        tiles = tuple(tiles or self.TILES)
        times = {}
        for k in buckets:
            n = int(round(2.0 ** (k + 0.5)))
            count = max(2, points_per_batch // n)
            probs = [datagen.gaussian_mixture(seed * 1000 + 100 * k + i, n) for i in range(count)]
            coords = [p[0] for p in probs]
            q = np.ascontiguousarray(np.concatenate([p[1] for p in probs]), np.float64)
            tl = {leaf: self._time_batch(coords, q, leaf, 8, degree, theta, eps, kind, precision, reps)
                  for leaf in leaves}
            best_leaf = min(tl, key=tl.get)
            ts = {8: tl[best_leaf]}
            for sp in splits:
                if sp not in ts:
                    ts[sp] = self._time_batch(coords, q, best_leaf, sp, degree, theta, eps, kind, precision, reps)
            best_split = min(ts, key=ts.get)
            tt = {256: ts[best_split]}
            for tile in tiles:
                if tile not in tt:
                    tt[tile] = self._time_batch(coords, q, best_leaf, best_split, degree, theta, eps, kind, precision,
                                                reps, tile)
            best_tile = min(tt, key=tt.get)
            self.table[k] = (best_leaf, best_split, best_tile)
            times[k] = {"n": n, "problems": count, "leaf_ms": tl, "split_ms": ts, "tile_ms": tt}
            if log:
                log(f"bucket 2^{k}: n={n} x{count}: leaf {best_leaf} split {best_split} tile {best_tile} "
                    f"({tt[best_tile]:.2f} ms; leaves {', '.join(f'{a}:{b:.2f}' for a, b in tl.items())})")
        self.meta = {"degree": degree, "theta": theta, "eps": eps, "kind": kind, "precision": precision,
                     "points_per_batch": points_per_batch, "times_ms": {str(k): v for k, v in times.items()}}
        return self
