"""Plain FP64 solves at the benchmark configurations' full sizes against the
reference library, on sampled target leaves.

A whole reference solve of these workloads takes minutes to an hour on the
host cores, so the reference (its own sources, OpenMP) runs its full upward
pass, then its own interaction routines (poisson_fmm_interactions_3d,
poisson_vel_fmm_interactions_3d) on the pairs whose target panel is a sampled
leaf or one of its ancestors, then its parent_to_child / leaf_to_point
functors along those panels (the fixed downward pass: leaves above the last
level receive their far field). The targets of the sampled leaves then carry
the reference's complete result, which the GPU's full solve must match to
relative L2 <= 1e-12 (src/fmm_interactions/poisson_fmm_impl.hpp:211-442,
poisson_vel_fmm_impl.hpp:10-257, src/downward_pass.cpp:7-41).

Workloads (tree, lists and leaf indices are bit-identical on both sides;
the test checks the panel count and the sampled leaves' point counts):
* 3-D uniform cube, N = 1,048,576, n = 8, theta 0.7, leaf 2000, eps 1e-4:
  the potential of the potential + gradient solve, and the vector kernel.
  Sampled: leaves on level 3 (about 2,000 points each: several target tiles,
  split source lists) and on level 4.
* 3-D Plummer sphere, N = 4,194,304, n = 10, theta 0.7, leaf 2000: potential
  (leaves on levels 2, 5, 7 and 9).
* Unit-sphere surface, N = 2,097,152, n = 10, theta 0.8, eps 1e-3: the
  vector kernel.
"""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-12


def rel(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.fixture(scope="module")
def ref_threads():
    from oracle import RefLib
    if not RefLib.available():
        pytest.skip("reference library oracle/_ref/libbtkref.so not built")
    ref = RefLib(threads=os.cpu_count() or 1)
    yield ref
    ref.set_threads(1)


def pick_leaves(panels, per_level, seed):
    """Up to per_level[level] non-empty leaves of each listed level, seeded."""
    rng = np.random.default_rng(seed)
    out = []
    for lev, k in per_level.items():
        cand = np.flatnonzero((panels["is_leaf"] != 0) & (panels["level"] == lev) & (panels["point_count"] > 0))
        if len(cand):
            out.extend(rng.choice(cand, min(k, len(cand)), replace=False).tolist())
    return np.array(sorted(out), np.int32)


def check(ref, pts, q, degree, theta, eps, cases, per_level, seed):
    """cases: (GPU kind, reference kind, [(GPU component, reference component)])."""
    import torch

    import barytreek_b200 as btk
    rt = ref.create(3, pts, degree=degree, cluster_size=2000, theta=theta, eps=eps)
    leaves = pick_leaves(rt.trees[0]["panels"], per_level, seed)
    assert len(leaves) >= 2
    idx = rt.leaf_targets(leaves)
    qd = torch.from_numpy(q).cuda()
    for gkind, rkind, comps in cases:
        tc = btk.Treecode(pts, degree=degree, cluster_size=2000, theta=theta, eps=eps, kind=gkind)
        assert tc.tree_t.panel_count == int(rt.info[1])
        assert np.array_equal(tc.tree_t.panels["point_count"][leaves], rt.trees[0]["panels"]["point_count"][leaves])
        out = tc.solve(qd).cpu().numpy()
        tc.close()
        r = rt.solve_leaves(rkind, q, leaves)
        for gc, rc in comps:
            e = rel(out[gc, idx], r[rc, idx])
            assert e <= TOL, (gkind, gc, e, leaves.tolist())


def test_uniform_1m_n8(ref_threads):
    import barytreek_b200 as btk
    from barytreek_b200 import datagen
    pts, q = datagen.uniform_box(1, 1 << 20, 3, 0.0, 1.0)
    check(ref_threads, pts, q, 8, 0.7, 1e-4,
          [(btk.KIND_FIELD, 0, [(0, 0)]), (btk.KIND_VEL, 1, [(0, 0), (1, 1), (2, 2)])],
          {3: 3, 4: 5}, seed=21)


def test_plummer_4m_n10(ref_threads):
    import barytreek_b200 as btk
    from barytreek_b200 import datagen
    pts, q = datagen.plummer(1, 1 << 22)
    check(ref_threads, pts, q, 10, 0.7, 1e-4, [(btk.KIND_POT, 0, [(0, 0)])], {2: 1, 5: 1, 7: 1, 9: 1}, seed=22)


def test_sphere_2m_vel_n10(ref_threads):
    import barytreek_b200 as btk
    from barytreek_b200 import datagen
    pts, q = datagen.sphere_surface(1, 1 << 21)
    check(ref_threads, pts, q, 10, 0.8, 1e-3, [(btk.KIND_VEL, 1, [(0, 0), (1, 1), (2, 2)])], {2: 1, 3: 1, 5: 2},
          seed=23)
