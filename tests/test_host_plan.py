"""Host-side parity (no GPU): meshes, entity numbering, dofmaps and the
sparsity pattern of the engine are bit-identical to the oracle's
restatement of DOLFIN; the row-gather plan is self-consistent."""
import numpy as np
import pytest

import dolfin_b200 as d2
from dolfin_b200 import _capi


def test_library_exports_every_header_symbol():
    import re, os
    hdr = open(os.path.join(os.path.dirname(__file__), "..", "include", "dolfin_b200.h")).read()
    declared = set(re.findall(r"\b(db2_[a-z0-9_]+)\s*\(", hdr))
    lib = _capi.lib()
    missing = [s for s in sorted(declared) if not hasattr(lib, s)]
    assert not missing, missing
    assert declared == set(_capi.exported_symbols())


@pytest.mark.parametrize("n", [(1, 1, 1), (2, 3, 4), (5, 4, 3)])
def test_unit_cube_mesh(orc, n):
    m = d2.UnitCubeMesh(*n)
    o = orc.unit_cube_mesh(*n)
    assert np.array_equal(m.cells(), o.cells)
    assert np.array_equal(m.coordinates(), o.coords)  # bit-exact coordinates


@pytest.mark.parametrize("diag", ["right", "left", "right/left", "left/right"])
def test_unit_square_mesh(orc, diag):
    m = d2.UnitSquareMesh(5, 7, diag)
    o = orc.unit_square_mesh(5, 7, diag)
    assert np.array_equal(m.cells(), o.cells)
    assert np.array_equal(m.coordinates(), o.coords)


@pytest.mark.parametrize("mesh,deg,vs", [("cube", 1, 1), ("cube", 2, 1), ("cube", 2, 3), ("cube", 1, 3),
                                         ("square", 1, 1), ("square", 2, 1)])
def test_dofmap_and_pattern_bit_exact(orc, mesh, deg, vs):
    if mesh == "cube":
        m, o = d2.UnitCubeMesh(3, 2, 4), orc.unit_cube_mesh(3, 2, 4)
    else:
        m, o = d2.UnitSquareMesh(6, 5), orc.unit_square_mesh(6, 5)
    V = d2.FunctionSpace(m, "Lagrange", deg, value_size=vs)
    od, N = orc.dofmap(o, deg, vs)
    assert V.dim() == N
    assert np.array_equal(V.dofmap().cell_dofs_all(), od)
    rp, cols = V.pattern().csr_host()
    orp, ocols = orc.sparsity(N, N, od, od)
    assert np.array_equal(rp, orp)
    assert np.array_equal(cols, ocols)


def test_edges_match_key_numbering(orc):
    m = d2.UnitCubeMesh(3, 3, 2)
    o = orc.unit_cube_mesh(3, 3, 2)
    ce, ev = orc.edges(o)
    assert m.num_edges() == ev.shape[0]


@pytest.mark.parametrize("tdim,deg", [(3, 1), (3, 2), (2, 1), (2, 2)])
def test_plan_slots_point_at_the_relabelled_nodes(tdim, deg):
    """Every (node row, cell) incidence's slot bytes point at the columns of
    the cell's nodes in the canonical relabelled order."""
    m = d2.UnitCubeMesh(2, 2, 2) if tdim == 3 else d2.UnitSquareMesh(4, 3)
    V = d2.FunctionSpace(m, "Lagrange", deg)
    plan = V.pattern().plan()
    cd = V.dofmap().cell_dofs_all()
    k = cd.shape[1]
    nv = tdim + 1
    E = [(2, 3), (1, 3), (1, 2), (0, 3), (0, 2), (0, 1)] if tdim == 3 else [(1, 2), (0, 2), (0, 1)]
    rp, cols = plan["node_rowptr"], plan["node_cols"]
    for node in range(V.dim()):
        incs = plan["inc"][plan["inc_ptr"][node]:plan["inc_ptr"][node + 1]]
        cells = incs & 0x0FFFFFFF
        assert np.all(np.diff(cells.astype(np.int64)) > 0)  # ascending cell order
        for s, w in zip(range(plan["inc_ptr"][node], plan["inc_ptr"][node + 1]), incs):
            c, li = int(w & 0x0FFFFFFF), int(w >> 28)
            assert cd[c, li] == node
            first = [li] if li < nv else list(E[li - nv])
            perm = first + [a for a in range(nv) if a not in first]
            local = list(perm)
            if deg == 2:
                for (A, B) in E:
                    p, q = sorted((perm[A], perm[B]))
                    local.append(nv + E.index((p, q)))
            slots = plan["pos"][s][:k]
            row = cols[rp[node]:rp[node + 1]]
            assert [int(row[x]) for x in slots] == [int(cd[c, j]) for j in local]


def test_tiles_cover_rows_once():
    m = d2.UnitCubeMesh(3, 3, 3)
    V = d2.VectorFunctionSpace(m, "Lagrange", 2)
    plan = V.pattern().plan()
    t = plan["tiles"]
    t = t[np.lexsort((t[:, 1], t[:, 0]))]
    nn = V.dim() // 3
    for c in range(3):
        tc = t[t[:, 0] == c]
        assert tc[0, 1] == 0 and tc[-1, 2] == nn
        assert np.all(tc[1:, 1] == tc[:-1, 2])
        assert np.all(tc[:, 2] > tc[:, 1])


def test_errors_are_raised_not_crashed():
    with pytest.raises(_capi.DB2Error):
        d2.Mesh(np.zeros((3, 2)), np.array([[0, 2, 1]], np.uint32))  # unordered cell
    with pytest.raises(_capi.DB2Error):
        d2.Mesh(np.zeros((3, 2)), np.array([[0, 1, 5]], np.uint32))  # index out of range
    m = d2.UnitSquareMesh(2, 2)
    with pytest.raises(_capi.DB2Error):
        d2.FunctionSpace(m, "Lagrange", 3)
    with pytest.raises(NotImplementedError):
        d2.FunctionSpace(m, "DG", 1)


def test_recogniser_identifies_named_forms():
    from dolfin_b200.ufl import recognise
    m = d2.UnitCubeMesh(1, 1, 1)
    V = d2.FunctionSpace(m, "Lagrange", 2)
    W = d2.FunctionSpace(m, "Lagrange", 1)
    u, v = d2.TrialFunction(V), d2.TestFunction(V)
    import torch
    kappa = d2.Function(W)
    r = recognise(kappa * d2.inner(d2.grad(u), d2.grad(v)) * d2.dx)
    assert r.kind == _capi.FORM_DIFFUSION and r.coeff == _capi.COEFF_P1 and r.function is kappa
    r = recognise(d2.dot(d2.grad(v), 3.0 * d2.grad(u)) * d2.dx)
    assert r.coeff == _capi.COEFF_CONSTANT and r.constant[0] == 3.0
    r = recognise(kappa * v * d2.dx)
    assert r.kind == _capi.FORM_LOAD and r.coeff == _capi.COEFF_P1
    VV = d2.VectorFunctionSpace(m, "Lagrange", 2)
    u, v = d2.TrialFunction(VV), d2.TestFunction(VV)
    E, nu = 1.0, 0.3
    mu, lmbda = d2.Constant(E / (2 * (1 + nu))), d2.Constant(E * nu / ((1 + nu) * (1 - 2 * nu)))
    eps = lambda w: d2.sym(d2.grad(w))
    sigma = lambda w: 2 * mu * eps(w) + lmbda * d2.tr(eps(w)) * d2.Identity(3)
    r = recognise(d2.inner(sigma(u), eps(v)) * d2.dx)
    assert r.kind == _capi.FORM_ELASTICITY
    assert r.mu == float(mu) and r.lmbda == float(lmbda)
    r = recognise(d2.inner(d2.Constant((0.0, 0.0, -1.0)), v) * d2.dx)
    assert r.kind == _capi.FORM_LOAD and r.constant == (0.0, 0.0, -1.0)
    with pytest.raises(NotImplementedError):
        recognise(u[0] * v[0] * d2.dx)
