"""Partitioning a frequency sweep of independent matrices across GPUs.

The matrices of a sweep are independent, so a sweep shards across ranks with
no exchange on the data path: each rank (one process per GPU) takes a subset,
runs the batched algorithm on it, and the results come back to one host.
The subsets are chosen by LPT (longest processing time first): matrices in
decreasing cost, each to the rank with the least work so far. The cost of
one exponential is n^3 (s + 8) -- about its product count at Pade degree 13
times n^3 -- with s estimated before any matrix exists from the frequency:
A = -(G + i w C) has ||A||_1 close to w ||C||_1, so s grows as log2(w).

No counterpart in the reference, which runs on one machine's CPU cores
(src/Tensile/MatrixExponential.cs processes one matrix per call).
"""
from __future__ import annotations

import math


def expm_cost_estimate(n: int, omega: float) -> float:
    """n^3 (s + 8), with s estimated as log2(max(w, 1)): a ranking cost, not
    a prediction of the squarings."""
    s = math.log2(max(float(omega), 1.0))
    return float(n) ** 3 * (s + 8.0)


def lpt_partition(costs, ranks: int):
    """Indices of `costs` split over `ranks` ranks by LPT: descending cost,
    each to the least-loaded rank (ties to the lowest rank). Returns one index
    list per rank, each in increasing index order, and the ranks' loads."""
    if ranks < 1:
        raise ValueError("at least one rank")
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    parts = [[] for _ in range(ranks)]
    loads = [0.0] * ranks
    for i in order:
        r = min(range(ranks), key=lambda q: (loads[q], q))
        parts[r].append(i)
        loads[r] += float(costs[i])
    return [sorted(p) for p in parts], loads


def gather_to_rank0(dist, rank: int, world: int, indices, results):
    """Collect every rank's (index, result) pairs on rank 0 through the
    process group's host-side object gather (gloo, or NCCL with the objects
    staged through the CPU). Returns the results in index order on rank 0,
    None elsewhere. Every rank must call it."""
    mine = list(zip(indices, results))
    if world == 1:
        return [r for _, r in sorted(mine, key=lambda x: x[0])]
    box = [None] * world if rank == 0 else None
    dist.gather_object(mine, box, dst=0)
    if rank != 0:
        return None
    merged = [pair for part in box for pair in part]
    merged.sort(key=lambda x: x[0])
    return [r for _, r in merged]
