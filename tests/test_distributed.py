"""Multi-process plumbing on CPU (gloo, world size 2, 127.0.0.1).

Each rank takes its size-balanced share of a batch of small independent
problems, evaluates them (the oracle's FP64 direct sum stands in for the
solve, which needs a GPU), and rank 0 gathers the outputs in problem order;
the result must equal the single-process evaluation. The max and sum
reductions must agree with the ranks' local values.
"""
import os
import socket

import numpy as np
import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _problems():
    from barytreek_b200 import datagen
    sizes = [120, 40, 300, 75, 210, 33, 90]
    return [datagen.gaussian_mixture(50 + b, n) for b, n in enumerate(sizes)]


def _solve_all(oracle, probs, which):
    outs = []
    for b in which:
        pts, q = probs[b]
        outs.append(oracle.direct(3, 0, 1e-4, pts, pts, q))
    return np.concatenate(outs, axis=1) if outs else np.zeros((1, 0))


def _worker(rank, world, port, result_path):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime

    import torch.distributed as dist

    from barytreek_b200 import distributed as D
    from oracle import Oracle
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        probs = _problems()
        sizes = [len(p[1]) for p in probs]
        offs = np.zeros(len(sizes) + 1, np.int64)
        offs[1:] = np.cumsum(sizes)
        mine = D.shard_problems(sizes, world)[rank]
        local = _solve_all(Oracle(), probs, mine)
        full = D.gather_problem_outputs(local, mine, offs, int(offs[-1]))
        mx = D.reduce_over_ranks(float(rank + 1), "max")
        sm = D.reduce_over_ranks(float(len(mine)), "sum")
        if rank == 0:
            np.savez(result_path, full=full, mx=mx, sm=sm)
    finally:
        dist.destroy_process_group()


def test_shard_is_balanced_partition():
    from barytreek_b200.distributed import shard_problems
    sizes = np.random.default_rng(0).integers(4096, 262144, 256)
    for world in (1, 2, 3, 8):
        parts = shard_problems(sizes, world)
        flat = sorted(b for p in parts for b in p)
        assert flat == list(range(len(sizes)))
        loads = [sum(int(sizes[b]) for b in p) for p in parts]
        assert max(loads) - min(loads) <= int(max(sizes))


def test_two_ranks_gloo(tmp_path, oracle):
    import torch.multiprocessing as mp
    path = str(tmp_path / "r.npz")
    mp.spawn(_worker, args=(2, _free_port(), path), nprocs=2, join=True)
    z = np.load(path)
    probs = _problems()
    ref = _solve_all(oracle, probs, range(len(probs)))
    assert np.array_equal(z["full"], ref)
    assert float(z["mx"]) == 2.0 and float(z["sm"]) == len(probs)
