"""Generates the golden fixtures in tests/golden/ from the reference itself.

The reference ships no tests or golden vectors (its examples draw unseeded
random points and print a relative error), so the fixtures are produced by
running the reference's own code — its unmodified sources compiled against the
project's Kokkos-API host shim into oracle/_ref/libbtkref.so — on seeded inputs
from barytreek_b200.datagen. Each case stores the inputs, the reference's tree,
interaction lists and RunConfig, and every intermediate and final array of the
solve (downward pass with the two-site fix for leaves above the last level; the
unmodified downward pass where all leaves are on the last level), plus the
reference's direct sums.

Usage:  python tests/golden/gen_golden.py      (needs oracle/_ref/libbtkref.so)
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from barytreek_b200 import datagen  # noqa: E402
from oracle import RefLib  # noqa: E402

# name, dim, n, dist, seed, degree, leaf, theta, eps, kinds, n_sources
CASES = [
    ("ref2d_mixed", 2, 1500, "uniform", 1, 5, 40, 0.7, 1e-4, (0,), None),
    ("ref2d_lastlevel", 2, 4096, "uniform", 2, 6, 300, 0.7, 1e-4, (0,), None),
    ("ref3d_uniform", 3, 2000, "uniform", 3, 4, 60, 0.7, 1e-4, (0, 1), None),
    ("ref3d_plummer", 3, 2500, "plummer", 4, 4, 150, 0.7, 1e-4, (0, 1), None),
    ("ref3d_sphere", 3, 2000, "sphere", 5, 5, 80, 0.8, 1e-3, (1,), None),
    ("ref2d_split", 2, 1200, "uniform", 6, 5, 40, 0.7, 1e-4, (0,), 1000),
    ("ref3d_negative", 3, 1500, "negative", 7, 4, 60, 0.7, 1e-4, (0,), None),
]

NAMELISTS = {
    "nl_default": "interp_degree=8\ncluster_size=100\ntheta=0.7\nkernel_eps=1e-4\nend",
    "nl_clamp": "interp_degree=14\ncluster_size=0\ntheta=0.55\nkernel_eps=2.5e-3\nend",
    "nl_partial": "cluster_size=-5\ninterp_degree=3\nfoo=1\ntheta=0.1",
    "nl_eof": "interp_degree=5\ntheta=0.9\n",  # ends with a newline: the reference stops at EOF
}


def points(dist, seed, n, dim):
    if dist == "uniform":
        return datagen.uniform_box(seed, n, dim, -1.0, 1.0)
    if dist == "negative":  # all coordinates negative: exercises the max-init quirk
        return datagen.uniform_box(seed, n, dim, -3.0, -1.0)
    if dist == "plummer":
        return datagen.plummer(seed, n)
    return datagen.sphere_surface(seed, n)


def main():
    ref = RefLib(threads=1)
    for name, dim, n, dist, seed, deg, leaf, theta, eps, kinds, ns in CASES:
        pts, q = points(dist, seed, n, dim)
        src = None
        if ns is not None:
            src, q = datagen.uniform_box(seed + 100, ns, dim, -1.0, 1.0)
        rt = ref.create(dim, pts, src, degree=deg, cluster_size=leaf, theta=theta, eps=eps)
        data = {"params": np.array([dim, n, seed, deg, leaf, ns or 0], np.int64),
                "fparams": np.array([theta, eps]), "config": np.frombuffer(rt.config_bytes, np.uint8),
                "q": q, "all": rt.all}
        for d in range(dim):
            data[f"t{d}"] = pts[d]
            if src is not None:
                data[f"s{d}"] = src[d]
        for which, tag in ((0, "T"), (1, "S")):
            if which == 1 and src is None:
                continue
            tr = rt.trees[which]
            data[f"{tag}_panels"] = tr["panels"]
            data[f"{tag}_level_start"] = tr["level_start"]
            data[f"{tag}_leaf_of"] = tr["leaf_of"]
            data[f"{tag}_inside"] = tr["inside"]
        for k in ("pp", "pc", "cp", "cc"):
            data[k] = rt.lists[k]
        last_only = rt.leaves_on_last_level_only()
        data["last_level_only"] = np.array([int(last_only)])
        for kind in kinds:
            r = rt.solve(kind, q, fixed=True)
            for key, arr in r.items():
                data[f"k{kind}_{key}"] = arr
            if last_only:
                data[f"k{kind}_out_unfixed"] = rt.solve(kind, q, fixed=False)["out"]
            sources = src if src is not None else pts
            m = min(300, len(pts[0]))
            sub = tuple(c[:m] for c in pts)
            data[f"k{kind}_direct"] = ref.direct(dim, kind, eps, sub, sources, q)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **data)
        print(name, "panels", rt.info[1], "levels", rt.info[2], "lists", rt.info[5:9], "last-level-only", last_only)
    for name, text in NAMELISTS.items():
        path = os.path.join(HERE, name + ".txt")
        with open(path, "w") as f:
            f.write(text)
        out = {}
        for dim in (2, 3):
            out[f"cfg{dim}"] = np.frombuffer(ref.read_namelist(path, dim), np.uint8)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
        print(name)


if __name__ == "__main__":
    main()
