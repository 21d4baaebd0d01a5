"""One process per GPU: the plumbing around independent solves.

The treecode path itself has no data-path exchange on one problem (it runs on
one GPU). Two multi-GPU uses remain, neither with a collective in the data
path: N replicas of one solve (each rank its own problem), and a batch of
independent problems sharded by problem across ranks. This module holds the
host logic for both: a size-balanced assignment of problems to ranks, the
max/sum reductions of timings and counts over ranks (on the process group's
own device: CUDA tensors under NCCL, CPU tensors under gloo), and the gather of
per-rank results in problem order.
"""
from __future__ import annotations

import heapq

import numpy as np

__all__ = ["shard_problems", "world_info", "reduce_over_ranks", "gather_problem_outputs"]


def world_info():
    """(world size, rank) of the default process group, (1, 0) without one."""
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized():
        return dist.get_world_size(), dist.get_rank()
    return 1, 0


def shard_problems(sizes, world: int):
    """Assigns problems to ranks by the longest-processing-time rule on their
    point counts (largest first to the least loaded rank). Returns one sorted
    list of problem indices per rank; every problem appears exactly once."""
    if world < 1:
        raise ValueError("world must be >= 1")
    heap = [(0, r) for r in range(world)]
    out = [[] for _ in range(world)]
    for b in sorted(range(len(sizes)), key=lambda i: (-int(sizes[i]), i)):
        load, r = heapq.heappop(heap)
        out[r].append(b)
        heapq.heappush(heap, (load + int(sizes[b]), r))
    return [sorted(x) for x in out]


def _device():
    import torch
    import torch.distributed as dist
    return torch.device("cuda", torch.cuda.current_device()) if dist.get_backend() == "nccl" else torch.device("cpu")


def reduce_over_ranks(x: float, op: str = "max") -> float:
    """max or sum of a scalar over all ranks (x itself without a process group)."""
    import torch
    import torch.distributed as dist
    world, _ = world_info()
    if world == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=_device())
    dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max" else dist.ReduceOp.SUM)
    return float(t.item())


def gather_problem_outputs(local: np.ndarray, my_problems, offsets, total: int):
    """Assembles per-rank outputs ([ncomp, points of my problems] in the order
    of my_problems) into [ncomp, total] in problem order on rank 0 (None on the
    other ranks)."""
    import torch.distributed as dist
    world, rank = world_info()
    pieces = [(list(my_problems), np.ascontiguousarray(local))]
    if world > 1:
        gathered = [None] * world if rank == 0 else None
        dist.gather_object(pieces[0], gathered, dst=0)
        if rank != 0:
            return None
        pieces = gathered
    out = np.zeros((local.shape[0], total), dtype=local.dtype)
    for probs, arr in pieces:
        col = 0
        for b in probs:
            n = offsets[b + 1] - offsets[b]
            out[:, offsets[b]:offsets[b + 1]] = arr[:, col:col + n]
            col += n
    return out
