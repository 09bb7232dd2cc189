"""DirichletBC (dolfin/fem/DirichletBC.h) for the system assembler.

Boundary dofs are found topologically, as DirichletBC's default "topological"
method: the closure (vertices, and for P2 the edges) of the exterior facets
(facets with a single cell) that the marker accepts.  The values are applied
inside the assembly kernel by SystemAssembler::apply_bc's symmetric rule.
"""
from __future__ import annotations

import numpy as np

_TET_EDGES = [(2, 3), (1, 3), (1, 2), (0, 3), (0, 2), (0, 1)]
_TRI_EDGES = [(1, 2), (0, 2), (0, 1)]


def exterior_facets(cells):
    """(cell index, local facet index = opposite local vertex) of every facet
    that belongs to exactly one cell."""
    cells = np.asarray(cells, np.int64)
    nc, nv = cells.shape
    keys, owner, local = [], [], []
    for a in range(nv):
        f = np.delete(cells, a, axis=1)
        f.sort(axis=1)
        keys.append(f)
        owner.append(np.arange(nc))
        local.append(np.full(nc, a))
    keys = np.concatenate(keys)
    owner = np.concatenate(owner)
    local = np.concatenate(local)
    _, inv, counts = np.unique(keys, axis=0, return_inverse=True, return_counts=True)
    ext = counts[inv.ravel()] == 1
    return owner[ext], local[ext]


class DirichletBC:
    def __init__(self, V, value, where="on_boundary", method="topological"):
        if method != "topological":
            raise NotImplementedError("only the topological method is provided")
        self.V = V
        self.value = value
        self.where = where
        self._cache = None

    def function_space(self):
        return self.V

    def _marked_facets(self, mesh):
        cells = mesh.cells().astype(np.int64)
        x = mesh.coordinates()
        owner, local = exterior_facets(cells)
        if isinstance(self.where, str):
            if self.where != "on_boundary":
                raise NotImplementedError("markers: 'on_boundary' or a callable(x, on_boundary)")
            return owner, local
        keep = []
        for c, a in zip(owner, local):
            vs = np.delete(cells[c], a)
            pts = list(x[vs]) + [x[vs].mean(axis=0)]
            keep.append(all(bool(self.where(p, True)) for p in pts))
        keep = np.array(keep, bool)
        return owner[keep], local[keep]

    def dofs_and_values(self):
        if self._cache is not None:
            return self._cache
        V = self.V
        mesh = V.mesh()
        tdim = mesh.topology_dim()
        nv_cell = tdim + 1
        owner, local = self._marked_facets(mesh)
        cd = V.dofmap().cell_dofs_all()
        vs = V.value_size()
        k = cd.shape[1] // vs
        nn = V.dim() // vs
        # natural node numbers of the cells (vertices, then nv + edge index)
        if V.reordered():
            inv = np.argsort(V.node_numbers())
            nodes = inv[cd[:, :k] // vs]
        else:
            nodes = cd[:, :k]  # component-0 dofs are the node numbers
        bnodes = set()
        edges = _TET_EDGES if tdim == 3 else _TRI_EDGES
        for c, a in zip(owner, local):
            for b in range(nv_cell):
                if b != a:
                    bnodes.add(int(nodes[c, b]))
            if V.degree() == 2:
                for e, (p, q) in enumerate(edges):
                    if a not in (p, q):
                        bnodes.add(int(nodes[c, nv_cell + e]))
        bn = np.array(sorted(bnodes), np.int64)
        # coordinates of the boundary nodes (vertices or edge midpoints),
        # needed only for a callable value
        pts = None
        if callable(self.value):
            x = mesh.coordinates()
            allpts = np.zeros((nn, x.shape[1]))
            allpts[:mesh.num_vertices()] = x
            if V.degree() == 2:
                for e, (p, q) in enumerate(edges):
                    allpts[nodes[:, nv_cell + e]] = 0.5 * (x[nodes[:, p]] + x[nodes[:, q]])
            pts = allpts[bn]
        vals = self._values(pts, vs, bn.size)
        dofs = np.concatenate([V.node_dofs(c, bn) for c in range(vs)])
        values = np.concatenate([vals[:, c] for c in range(vs)])
        self._cache = (dofs, values)
        return self._cache

    def _values(self, pts, vs, n):
        from .function import Constant
        v = self.value
        if isinstance(v, Constant):
            v = v.values()
        if callable(v):
            out = np.array([np.atleast_1d(v(p)) for p in pts], np.float64).reshape(len(pts), -1)
        else:
            out = np.broadcast_to(np.atleast_1d(np.asarray(v, np.float64)), (n, vs)).copy()
        if out.shape[1] != vs:
            raise ValueError("DirichletBC value has the wrong size")
        return out
