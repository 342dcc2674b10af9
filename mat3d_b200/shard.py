"""Spreading a batch of RVE solves over the GPUs of one node (one process per
GPU, ``torch.distributed``).

The solves are independent (RVEs and load cases), so there is no data-path
collective: the work list is partitioned by device footprint, largest first
onto the least-loaded rank, each rank homogenizes its share, and the small
results (one C x C tensor per RVE) are gathered on the host at the end.
"""
from __future__ import annotations

import heapq

import numpy as np


def partition_by_footprint(costs, world):
    """Greedy largest-first assignment of items with the given costs onto
    ``world`` ranks (each item to the rank with the least total so far; ties
    to the lower rank).  Returns one sorted index list per rank."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    heap = [(0.0, r) for r in range(world)]
    heapq.heapify(heap)
    parts = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        parts[r].append(i)
        heapq.heappush(heap, (load + float(costs[i]), r))
    return [sorted(p) for p in parts]


def batch_costs(descs, precision="fp32_refine", kind=1, nload=6):
    """Device bytes of each batched-workload member (seed, N, vf, contrast)
    as one RVE with ``nload`` load cases; the work of a member scales the same way."""
    from . import footprint_bytes

    return [footprint_bytes(kind, (N, N, N), 0, precision, 1, nload) for _, N, _, _ in descs]


def gather_tensors(local_idx, local_tensors, n_total, group=None):
    """All-gather (host objects) the per-rank tensors into one (n_total, C, C)
    array ordered by global index; every rank gets the full result."""
    import torch.distributed as dist

    world = dist.get_world_size(group)
    mine = (list(local_idx), np.asarray(local_tensors))
    got = [None] * world
    dist.all_gather_object(got, mine, group=group)
    C = next(t.shape[-1] for _, t in got if len(t))
    out = np.full((n_total, C, C), np.nan)
    for idx, t in got:
        for i, m in zip(idx, t):
            out[i] = m
    return out
