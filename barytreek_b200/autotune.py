"""Runs the batch autotuner on this GPU and writes its table.

    python -m barytreek_b200.autotune --out barytreek_b200/autotune_table.json

For every size bucket 2^k <= N < 2^(k+1) (k = 12..17) it times batched solves
of representative Gaussian-mixture problems (3-D Coulomb potential, degree 6,
theta 0.6, mixed precision) at each candidate leaf size, then each work split
at the best leaf size, then each tile size (targets per work item) at the best
pair, and keeps the fastest (barytreek_b200.batch).
"""
from __future__ import annotations

import argparse

from .batch import DEFAULT_TABLE, Autotuner


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=DEFAULT_TABLE)
    ap.add_argument("--points-per-batch", type=int, default=1 << 20)
    ap.add_argument("--reps", type=int, default=3)
    args = ap.parse_args()
    t = Autotuner().tune(points_per_batch=args.points_per_batch, reps=args.reps, log=print)
    t.save(args.out)
    print(f"wrote {args.out}: {t.table}")


if __name__ == "__main__":
    main()
