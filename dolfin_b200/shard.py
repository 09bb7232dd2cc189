"""Sharding of assembly work over ranks (one process per GPU).

Assembly needs no data-path collective: a rank that owns a range of rows
assembles them completely from the cells around them (the incidence lists
are per row), and independent meshes are assigned whole.  Only the timing
(max over ranks) is reduced.
"""
from __future__ import annotations

import heapq

import numpy as np


def lpt_assign(weights, nranks):
    """Longest-processing-time assignment of independent items (e.g. meshes
    of a batch, weight = cells) to ranks; deterministic.  Returns a list of
    index lists, one per rank."""
    order = sorted(range(len(weights)), key=lambda i: (-weights[i], i))
    heap = [(0.0, r) for r in range(nranks)]
    heapq.heapify(heap)
    out = [[] for _ in range(nranks)]
    for i in order:
        load, r = heapq.heappop(heap)
        out[r].append(i)
        heapq.heappush(heap, (load + float(weights[i]), r))
    return [sorted(x) for x in out]


def row_partition(inc_ptr, nranks):
    """Split node rows into nranks contiguous ranges of near-equal work
    (incidences).  inc_ptr: the pattern's node -> incidence offsets.
    Returns an int array of nranks+1 node boundaries."""
    inc_ptr = np.asarray(inc_ptr, np.int64)
    total = inc_ptr[-1]
    targets = (np.arange(1, nranks) * total) // nranks
    cuts = np.searchsorted(inc_ptr, targets, side="left")
    return np.concatenate([[0], cuts, [len(inc_ptr) - 1]]).astype(np.int64)


def max_over_ranks(value, group=None):
    """Max of a per-rank scalar (e.g. device time in ms) over the process group."""
    import torch
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized():
        return float(value)
    backend = dist.get_backend(group)
    dev = "cuda" if backend == "nccl" else "cpu"
    t = torch.tensor([float(value)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())
