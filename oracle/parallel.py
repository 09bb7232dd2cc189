"""Row-block parallel driver of the CPU oracle.

TEST INFRASTRUCTURE ONLY: the correctness checker of the CUDA engine at the
benchmark sizes.  Only ``tests/`` imports this module; the product package
``dolfin_b200`` never does.

DOLFIN's serial assembly (dolfin/fem/Assembler.cpp:148-193 with the
EigenMatrix::add scatter, dolfin/la/EigenMatrix.cpp:156-166) adds every
cell's element tensor into the rows of its dofs in cell order.  A row's
values therefore depend only on the cells incident to it, visited in
ascending cell order.  This driver splits the node rows into contiguous
blocks; a worker process takes the cells incident to its block (ascending),
runs the oracle's own sparsity (SparsityPatternBuilder.cpp:94-111 restated)
and cell loop on that sub-mesh with the full-size dofmap, and keeps only its
block's rows, which are complete.  The pieces are exactly the rows the
oracle produces on the whole mesh, computed on all host cores.

Workers are started with the ``spawn`` method (safe after CUDA use) and
share inputs and outputs through ``multiprocessing.shared_memory``.
"""
from __future__ import annotations

import multiprocessing as mp
import os
from multiprocessing import shared_memory

import numpy as np


class _Shared:
    """numpy arrays in named shared memory, created by the parent."""

    def __init__(self):
        self.blocks = []
        self.desc = {}

    def put(self, name, arr):
        arr = np.ascontiguousarray(arr)
        shm = shared_memory.SharedMemory(create=True, size=max(arr.nbytes, 1))
        view = np.ndarray(arr.shape, arr.dtype, buffer=shm.buf)
        view[...] = arr
        self.blocks.append(shm)
        self.desc[name] = (shm.name, arr.shape, arr.dtype.str)
        return view

    def empty(self, name, shape, dtype, fill=0):
        shm = shared_memory.SharedMemory(create=True, size=max(int(np.prod(shape)) * np.dtype(dtype).itemsize, 1))
        view = np.ndarray(shape, dtype, buffer=shm.buf)
        view[...] = fill
        self.blocks.append(shm)
        self.desc[name] = (shm.name, tuple(shape), np.dtype(dtype).str)
        return view

    def close(self):
        for shm in self.blocks:
            shm.close()
            shm.unlink()
        self.blocks = []


def _attach(desc):
    out, handles = {}, []
    for name, (shm_name, shape, dt) in desc.items():
        shm = shared_memory.SharedMemory(name=shm_name)
        handles.append(shm)
        out[name] = np.ndarray(shape, np.dtype(dt), buffer=shm.buf)
    return out, handles


def _form(orc, spec):
    if spec is None:
        return None
    kw = dict(spec)
    kind = kw.pop("kind")
    tdim = kw.pop("tdim")
    return orc.form(kind, tdim, **kw)


def _worker(task):
    """Rows of nodes [n0, n1) (every component) from their incident cells."""
    from oracle import oracle as orc
    desc, meta, n0, n1 = task
    a, handles = _attach(desc)
    try:
        tdim, N, bs, k_node = meta["tdim"], meta["N"], meta["bs"], meta["k_node"]
        nn = N // bs
        dofs = a["dofs"]
        nodes = dofs[:, :k_node]  # component-0 dofs are the node numbers (natural numbering)
        sel = np.nonzero(((nodes >= n0) & (nodes < n1)).any(axis=1))[0]
        sub = orc.Mesh(tdim, a["coords"], np.ascontiguousarray(a["cells"][sel]))
        dsub = np.ascontiguousarray(dofs[sel])
        rp, cols = orc.sparsity(N, N, dsub, dsub)
        fa, fl = _form(orc, meta["a"]), _form(orc, meta["L"])
        vals = orc.assemble_matrix(fa, sub, dsub, dsub, rp, cols,
                                   w=a.get("wa"), w2=a.get("wa2")) if fa is not None else None
        b = orc.assemble_vector(fl, sub, dsub, N, w=a.get("wL")) if fl is not None else None
        erp = a["rowptr"]
        bad = 0
        for c in range(bs):
            r0, r1 = c * nn + n0, c * nn + n1
            if b is not None:
                a["b"][r0:r1] = b[r0:r1]
            if vals is None:
                continue
            if not np.array_equal(np.diff(rp[r0:r1 + 1]), np.diff(erp[r0:r1 + 1])):
                bad += int(np.count_nonzero(np.diff(rp[r0:r1 + 1]) != np.diff(erp[r0:r1 + 1])))
                continue
            a["cols"][erp[r0]:erp[r1]] = cols[rp[r0]:rp[r1]]
            a["vals"][erp[r0]:erp[r1]] = vals[rp[r0]:rp[r1]]
        return bad, int(sel.size)
    finally:
        for h in handles:
            h.close()


def node_blocks(nn, nblocks, split=None):
    """Contiguous node ranges; P2 spaces (split = number of vertices) never
    mix vertex and edge nodes in one block, which keeps each block's cells a
    compact slab of the structured mesh."""
    parts = [(0, nn)] if split is None or split >= nn else [(0, split), (split, nn)]
    out = []
    for lo, hi in parts:
        m = max(1, round(nblocks * (hi - lo) / nn))
        cuts = np.linspace(lo, hi, m + 1).astype(np.int64)
        out += [(int(cuts[i]), int(cuts[i + 1])) for i in range(m) if cuts[i + 1] > cuts[i]]
    return out


def default_procs():
    n = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)
    return max(1, min(n, 32))


def assemble_rows(mesh, dofs, N, bs, k_node, rowptr, a=None, L=None, wa=None, wa2=None, wL=None,
                  nvert=None, procs=None, blocks_per_proc=2):
    """The oracle's CSR values and vector on the whole mesh, by row blocks.

    mesh: oracle.Mesh; dofs: natural cell dofmap (C x k); rowptr: the CSR
    row pointers to lay the values out on (the engine's, which the oracle's
    own row lengths are checked against).  a / L: oracle form parameters as
    dicts (kind, tdim, degree0, vsize0, coeff, c, mu, lmbda).

    Returns (cols, vals, b, mismatched_rows, cells_visited): cols/vals in the
    given rowptr layout (rows whose oracle length differs are counted in
    mismatched_rows and left zero), b (or None)."""
    procs = procs or default_procs()
    sh = _Shared()
    try:
        sh.put("coords", np.asarray(mesh.coords, np.float64))
        sh.put("cells", np.asarray(mesh.cells, np.uint32))
        sh.put("dofs", np.asarray(dofs, np.int32))
        sh.put("rowptr", np.asarray(rowptr, np.int64))
        for name, w in (("wa", wa), ("wa2", wa2), ("wL", wL)):
            if w is not None:
                sh.put(name, np.asarray(w, np.float64))
        nnz = int(rowptr[-1])
        cols = sh.empty("cols", (nnz if a is not None else 1,), np.int32, fill=-1)
        vals = sh.empty("vals", (nnz if a is not None else 1,), np.float64)
        b = sh.empty("b", (N if L is not None else 1,), np.float64)
        meta = dict(tdim=mesh.tdim, N=int(N), bs=int(bs), k_node=int(k_node), a=a, L=L)
        blocks = node_blocks(N // bs, procs * blocks_per_proc, nvert)
        tasks = [(sh.desc, meta, n0, n1) for n0, n1 in blocks]
        ctx = mp.get_context("spawn")
        with ctx.Pool(min(procs, len(tasks))) as pool:
            res = pool.map(_worker, tasks, chunksize=1)
        bad = sum(r[0] for r in res)
        visited = sum(r[1] for r in res)
        return (cols.copy() if a is not None else None, vals.copy() if a is not None else None,
                b.copy() if L is not None else None, bad, visited)
    finally:
        sh.close()
