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


def row_block_dofs(nnodes, bs, node_begin, node_end):
    """Global dof numbers of a row block (natural numbering), in the order
    the block stores them: component-major, nodes ascending."""
    nodes = np.arange(node_begin, node_end, dtype=np.int64)
    return np.concatenate([c * nnodes + nodes for c in range(bs)])


class RowBlock:
    """One rank's share of a single-mesh assembly: the CSR rows and b entries
    of nodes [node_begin, node_end) (every component), assembled from the
    cells around them and held alone -- the rank allocates its block, not
    the whole matrix.  The row-owner counterpart of DOLFIN's distributed
    SparsityPattern (dolfin/la/SparsityPattern.cpp:200-255): ranks exchange
    nothing, since no rank produces entries of rows it does not own.

        blk = RowBlock(V, n0, n1)
        blk.assemble_system(a, L)       # blk.vals, blk.b (device, local)
    """

    def __init__(self, V, node_begin, node_end, keep_diagonal=False):
        import torch
        self.V = V
        self.pattern = V.pattern(keep_diagonal)
        self.node_begin, self.node_end = int(node_begin), int(node_end)
        self.pattern.set_row_block(self.node_begin, self.node_end)
        self.nrows, self.nnz = self.pattern.row_block_info()
        self.vals = torch.empty(self.nnz, dtype=torch.float64, device="cuda")
        self.b = torch.empty(self.nrows, dtype=torch.float64, device="cuda")

    def dofs(self):
        """Global dofs of the block's rows (its b entries), in block order."""
        nn = self.V.dim() // self.V.value_size()
        return row_block_dofs(nn, self.V.value_size(), self.node_begin, self.node_end)

    def csr_host(self):
        return self.pattern.row_block_csr_host()

    def assemble_system(self, a, L, bcs=None, precision="fp64"):
        """SystemAssembler(a, L, bcs) restricted to the block's rows."""
        from .assembling import SystemAssembler
        S = SystemAssembler(a, L, bcs, precision)
        if S.ra.V is not self.V:
            raise RuntimeError("the forms live on another function space")
        S.assemble_into(self.pattern, self.vals, self.b)
        return self.vals, self.b

    def release(self):
        """Back to whole-pattern assembly (all rows, whole tensors)."""
        self.pattern.set_row_range(0, self.V.dim() // self.V.value_size())


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
