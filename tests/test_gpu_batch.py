"""Batched solves on the GPU: one forest plan, one captured graph.

* FP64 batch vs each problem solved alone by its own plan (the plan path the
  parity tests pin to the reference): relative L2 <= 1e-13 per problem (the
  same arithmetic; only the order of split-item atomics differs), and one
  problem against the reference library itself (<= 1e-12).
* Mixed-precision batch (FP32 bulk, FP64 final sums) against the FP64 direct
  sum at sampled targets of every problem: relative L2 <= 1e-6.
* Graph replay: a second solve with other charges matches its eager
  single-problem solves; the captured graph holds a handful of kernels, with
  one interaction launch for all problems.
* The autotuner returns a leaf size and work split for each bucket it tunes.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b)))


def _probs(seed, sizes):
    from barytreek_b200 import datagen
    return [datagen.gaussian_mixture(seed + b, n) for b, n in enumerate(sizes)]


SIZES = [4096, 23000, 5300, 61000, 9000, 17000, 4500, 31000]
LEAVES = [256, 512, 256, 1024, 256, 512, 128, 512]


def test_fp64_batch_matches_single_plans_and_reference(reflib):
    import barytreek_b200 as btk
    from barytreek_b200.batch import Batch
    probs = _probs(300, SIZES)
    coords = [p[0] for p in probs]
    q = np.concatenate([p[1] for p in probs])
    b = Batch(coords, degree=6, theta=0.6, eps=1e-4, kind=btk.KIND_POT, precision=btk.PREC_FP64,
              cluster_size=LEAVES, work_split=8)
    out = b.solve(q).cpu().numpy()
    for i, (pts, qi) in enumerate(probs):
        tc = btk.Treecode(pts, degree=6, cluster_size=LEAVES[i], theta=0.6, eps=1e-4, kind=btk.KIND_POT)
        one = tc.solve(qi).cpu().numpy()
        assert rel(out[:, b.offsets[i]:b.offsets[i + 1]], one) <= 1e-13, i
    # problem 1 against the reference treecode
    pts, qi = probs[1]
    rt = reflib.create(3, pts, degree=6, cluster_size=LEAVES[1], theta=0.6, eps=1e-4)
    ref = rt.solve(0, qi, fixed=True)["out"]
    assert rel(out[0, b.offsets[1]:b.offsets[2]], ref[0]) <= 1e-12
    st = b.stats()
    assert st["n_problems"] == len(SIZES) and st["total_points"] == sum(SIZES)
    assert 0 < st["graph_kernel_nodes"] <= 40, st


def test_mixed_batch_accuracy_and_replay(oracle):
    import torch

    import barytreek_b200 as btk
    from barytreek_b200.batch import Batch
    probs = _probs(500, SIZES)
    coords = [p[0] for p in probs]
    q = np.concatenate([p[1] for p in probs])
    b = Batch(coords, degree=6, theta=0.6, eps=1e-4, kind=btk.KIND_POT, precision=btk.PREC_MIXED,
              cluster_size=LEAVES, work_split=8)
    out = b.solve(q).cpu().numpy()
    rng = np.random.default_rng(5)
    for i, (pts, qi) in enumerate(probs):
        idx = rng.choice(len(qi), size=min(300, len(qi)), replace=False)
        ds = oracle.direct(3, 0, 1e-4, tuple(c[idx] for c in pts), pts, qi)
        assert rel(out[0, b.offsets[i] + idx], ds[0]) <= 1e-6, i
    # replay with new charges equals eager single-problem mixed solves
    q2 = np.concatenate([np.sin(3.0 * np.arange(len(p[1]))) for p in probs])
    out2 = b.solve(torch.from_numpy(q2).cuda()).cpu().numpy()
    for i, (pts, _) in enumerate(probs):
        tc = btk.Treecode(pts, degree=6, cluster_size=LEAVES[i], theta=0.6, eps=1e-4, kind=btk.KIND_POT,
                          precision=btk.PREC_MIXED)
        one = tc.solve(q2[b.offsets[i]:b.offsets[i + 1]]).cpu().numpy()
        assert rel(out2[:, b.offsets[i]:b.offsets[i + 1]], one) <= 1e-12, i
    assert b.stats()["last_ms"] > 0


def test_autotuner_picks_per_bucket():
    from barytreek_b200.batch import Autotuner
    t = Autotuner().tune(buckets=[12, 14], points_per_batch=1 << 16, leaves=(128, 512), splits=(4, 8), reps=1)
    for k in (12, 14):
        leaf, split, tile = t.table[k]
        assert leaf in (128, 512) and split in (4, 8) and tile in (128, 256)
    assert t.leaf_for(5000) == t.table[12][0]
    assert t.tile_for_batch([5000] * 5 + [20000]) == t.table[12][2]  # bucket 2^12 holds most points
