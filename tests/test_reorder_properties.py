"""reorder_dofs_serial = True: the reverse Cuthill-McKee numbering checked by
its defining properties, in a restatement of its own (plain Python over a
node graph rebuilt from the cells), on the meshes of DOLFIN's own dofmap
tests (python/test/unit/fem/test_dofmap.py: UnitSquareMesh(4, 4),
UnitCubeMesh(2, 2, 2)) and larger ones.  With cm the visiting order (the
k-th visited node gets number n-1-k):

* every node is numbered once;
* BFS levels: when cm[p] is dequeued, its not yet queued neighbours are
  exactly the next block of cm;
* degree order: each block is sorted by degree, ascending;
* ties: equal degrees stay in dolfin::Set insertion order (the order in
  which the parent's neighbours were first inserted, cell by cell).  Boost
  sorts each block with std::sort, which is not stable; but every block on
  these meshes holds at most 16 nodes, and std::sort (libstdc++, whose
  threshold is 16; other libraries use larger ones) sorts such ranges by
  insertion sort, which is stable -- so the numbering does not depend on
  how the library's introsort orders ties, and the test checks that bound;
* starts: each connected component starts at the node Boost's
  find_starting_node reaches from the component's lowest-numbered node
  (repeated BFS to the minimum-degree node of the last level, the first
  visited on ties, while the eccentricity grows).
Host only."""
import numpy as np
import pytest

import dolfin_b200 as d2

INSERTION_SORT_MAX = 16


@pytest.fixture
def reordered():
    old = d2.parameters["reorder_dofs_serial"]
    d2.parameters["reorder_dofs_serial"] = True
    yield
    d2.parameters["reorder_dofs_serial"] = old


def _set_graph(cell_nodes, nn):
    """Neighbour lists in dolfin::Set insertion order: for each cell, each
    ordered pair (i, j), i != j, of its nodes in local order, j appended to
    i's list unless already there (DofMapBuilder.cpp compute_node_reordering)."""
    nbr = [dict() for _ in range(nn)]
    for row in cell_nodes:
        row = [int(a) for a in row]
        for a in row:
            for b in row:
                if a != b:
                    nbr[a].setdefault(b, None)
    return [list(d) for d in nbr]


def _bfs_last_level(nbr, deg, s):
    """(eccentricity of s, the first minimum-degree node of the last BFS
    level in visit order, the nodes reached)."""
    seen = {s}
    level = [s]
    ecc = 0
    while True:
        nxt = []
        for x in level:
            for y in nbr[x]:
                if y not in seen:
                    seen.add(y)
                    nxt.append(y)
        if not nxt:
            break
        level = nxt
        ecc += 1
    best = level[0]
    for x in level[1:]:
        if deg[x] < deg[best]:
            best = x
    return ecc, best, seen


def _starting_node(nbr, deg, r):
    er, x, comp = _bfs_last_level(nbr, deg, r)
    ex, y, _ = _bfs_last_level(nbr, deg, x)
    while ex > er:
        r, er, x = x, ex, y
        ex, y, _ = _bfs_last_level(nbr, deg, x)
    return x, comp


@pytest.mark.parametrize("tdim,n,deg,vs", [(2, 4, 1, 1), (2, 4, 2, 1), (3, 2, 1, 1), (3, 2, 2, 1),
                                           (3, 2, 2, 3), (2, 6, 1, 1), (2, 5, 2, 1), (3, 3, 1, 1),
                                           (3, 4, 2, 1), (3, 6, 2, 1), (2, 24, 2, 2)])
def test_rcm_numbering_has_the_cuthill_mckee_properties(reordered, tdim, n, deg, vs):
    m = d2.UnitSquareMesh(n, n) if tdim == 2 else d2.UnitCubeMesh(n, n, n)
    V = d2.FunctionSpace(m, "Lagrange", deg, value_size=vs)
    new = np.asarray(V.node_numbers())
    nn = new.size
    assert np.array_equal(np.sort(new), np.arange(nn))
    # natural node numbers of the cells: a cell's dofs are component-major,
    # dof = vs * node + component
    inv = np.argsort(new)
    cd = np.asarray(V.dofmap().cell_dofs_all())
    cell_nodes = inv[cd[:, :cd.shape[1] // vs] // vs]
    nbr = _set_graph(cell_nodes, nn)
    degree = [len(x) for x in nbr]
    cm = [int(x) for x in inv[::-1]]  # cm[k] = node numbered n-1-k
    queued = np.zeros(nn, bool)
    tail = 0
    for p in range(nn):
        u = cm[p]
        if p == tail:  # queue empty: u starts a new component
            comp_first = min(_bfs_last_level(nbr, degree, u)[2])
            start, comp = _starting_node(nbr, degree, comp_first)
            assert u == start and u in comp
            queued[u] = True
            tail += 1
        assert queued[u]
        fresh = [v for v in nbr[u] if not queued[v]]  # Set insertion order
        assert len(fresh) <= INSERTION_SORT_MAX
        block = cm[tail:tail + len(fresh)]
        assert block == sorted(fresh, key=lambda v: degree[v])  # stable: ties in Set order
        queued[block] = True
        tail += len(fresh)
    assert tail == nn
