"""Host-side parity (no GPU): meshes, entity numbering, dofmaps and the
sparsity pattern of the engine are bit-identical to the oracle's
restatement of DOLFIN; the row-gather plan is self-consistent."""
import os

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


def test_cpp_shim_library_loads_and_exports_the_assemblers():
    """libdolfin_b200_cpp.so (the C++ drop-in classes over the C ABI) loads
    beside the engine and defines GpuAssembler::assemble and the
    GpuSystemAssembler entry points declared in dolfin_b200_assembler.h."""
    import ctypes
    import subprocess
    lib = os.path.join(os.path.dirname(__file__), "..", "dolfin_b200", "_lib", "libdolfin_b200_cpp.so")
    _capi.lib()
    ctypes.CDLL(lib)
    syms = subprocess.run(["nm", "-DC", "--defined-only", lib], capture_output=True, text=True,
                          check=True).stdout
    for s in ["dolfin_b200::GpuAssembler::assemble(dolfin_b200::GenericTensor&, dolfin_b200::Form const&)",
              "dolfin_b200::GpuSystemAssembler::assemble(dolfin_b200::Matrix&, dolfin_b200::Vector&)",
              "dolfin_b200::GpuSystemAssembler::GpuSystemAssembler(",
              "dolfin_b200::DirichletBC::DirichletBC(",
              "dolfin_b200::forms::Elasticity("]:
        assert s in syms, s


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


@pytest.mark.parametrize("tdim,n", [(2, 6), (3, 3)])
def test_exterior_facets_match_oracle(orc, tdim, n):
    # facet-number (sorted key) order, cell and local facet of each
    m = d2.UnitSquareMesh(n, n) if tdim == 2 else d2.UnitCubeMesh(n, n, n)
    om = orc.unit_square_mesh(n, n) if tdim == 2 else orc.unit_cube_mesh(n, n, n)
    cell, local = m.exterior_facets()
    oc, ol = orc.exterior_facets(om)
    assert np.array_equal(cell, oc) and np.array_equal(local, ol)


def test_recogniser_facet_and_functional_parts():
    from dolfin_b200.ufl import recognise_functional, recognise_parts
    m = d2.UnitCubeMesh(1, 1, 1)
    V = d2.FunctionSpace(m, "Lagrange", 2)
    W = d2.FunctionSpace(m, "Lagrange", 1)
    u, v = d2.TrialFunction(V), d2.TestFunction(V)
    g = d2.Function(W)
    cell, facet = recognise_parts(d2.inner(d2.grad(u), d2.grad(v)) * d2.dx + 2.5 * g * u * v * d2.ds)
    assert cell.kind == _capi.FORM_DIFFUSION
    assert facet.kind == _capi.FORM_FACET_MASS and facet.coeff == _capi.COEFF_P1_SCALED
    assert facet.constant[0] == 2.5 and facet.function is g
    cell, facet = recognise_parts(g * v * d2.ds)
    assert cell is None and facet.kind == _capi.FORM_FACET_LOAD and facet.coeff == _capi.COEFF_P1
    VV = d2.VectorFunctionSpace(m, "Lagrange", 1)
    cell, facet = recognise_parts(d2.inner(d2.Constant((1.0, 0.0, -2.0)), d2.TestFunction(VV)) * d2.ds)
    assert facet.kind == _capi.FORM_FACET_LOAD and facet.constant == (1.0, 0.0, -2.0)
    x = d2.SpatialCoordinate(m)
    parts = recognise_functional(3.0 * x[2] * d2.dx(m) + d2.Constant(1.0) * d2.ds(m))
    assert parts[0][0] == _capi.FORM_FUNCTIONAL and parts[0][2] == _capi.COEFF_COORD
    assert parts[0][4][:2] == (3.0, 2.0)
    assert parts[1][0] == _capi.FORM_FACET_FUNCTIONAL and parts[1][4][0] == 1.0
    with pytest.raises(NotImplementedError):
        recognise_parts(d2.inner(d2.grad(u), d2.grad(v)) * d2.ds)
    with pytest.raises(NotImplementedError):
        d2.Constant(1.0) * d2.ds(m, subdomain_id=1)


@pytest.mark.parametrize("tdim,deg", [(2, 1), (2, 2), (3, 1), (3, 2)])
def test_facet_plan_slots_point_at_the_facet_nodes(orc, tdim, deg):
    import ctypes as C
    n = 3
    m = d2.UnitSquareMesh(n, n) if tdim == 2 else d2.UnitCubeMesh(n, n, n)
    om = orc.unit_square_mesh(n, n) if tdim == 2 else orc.unit_cube_mesh(n, n, n)
    V = d2.FunctionSpace(m, "Lagrange", deg)
    P = V.pattern()
    nb, ni, kf = C.c_int64(), C.c_int64(), C.c_int()
    _capi.call("db2_pattern_facet_plan_info", P.handle, C.byref(nb), C.byref(ni), C.byref(kf))
    bnode = np.empty(nb.value, np.uint32)
    bptr = np.empty(nb.value + 1, np.uint32)
    bverts = np.empty(ni.value * tdim, np.uint32)
    bslot = np.empty(ni.value * 8, np.uint8)
    ptr = lambda a: C.c_void_p(a.ctypes.data)
    _capi.call("db2_pattern_facet_plan_copy", P.handle, ptr(bnode), ptr(bptr), ptr(bverts), ptr(bslot))
    bverts, bslot, kf = bverts.reshape(-1, tdim), bslot.reshape(-1, 8), kf.value
    rp, cols = P.csr_host()
    od, N = orc.dofmap(om, deg)
    fc, fl = orc.exterior_facets(om)
    tet_e = [(2, 3), (1, 3), (1, 2), (0, 3), (0, 2), (0, 1)]
    tri_e = [(1, 2), (0, 2), (0, 1)]
    E = tet_e if tdim == 3 else tri_e
    facet_nodes, facet_verts = [], []
    for c, f in zip(fc, fl):
        vs = [a for a in range(tdim + 1) if a != f]
        nodes = {int(od[c, a]) for a in vs}
        if deg == 2:
            nodes |= {int(od[c, tdim + 1 + e]) for e, (p, q) in enumerate(E) if f not in (p, q)}
        facet_nodes.append(nodes)
        facet_verts.append({int(om.cells[c, a]) for a in vs})
    expect = {}
    for i, nodes in enumerate(facet_nodes):
        for nd in nodes:
            expect.setdefault(nd, []).append(i)
    assert sorted(expect) == bnode.tolist()
    nv = om.nv
    for t, node in enumerate(bnode):
        incs = list(range(bptr[t], bptr[t + 1]))
        assert len(incs) == len(expect[node])
        for s, i in zip(incs, expect[node]):  # facet-number order
            got = {int(cols[rp[node] + bslot[s, j]]) for j in range(kf)}
            assert got == facet_nodes[i]
            assert set(bverts[s].tolist()) == facet_verts[i]
            if node < nv:  # vertex row: canonical slot 0, relabelled vertex 0
                assert cols[rp[node] + bslot[s, 0]] == node and bverts[s, 0] == node
            else:          # edge row: canonical slot kf-1
                assert cols[rp[node] + bslot[s, kf - 1]] == node


def test_new_entry_points_reject_bad_arguments():
    # checked on the host before any device work: status codes, not crashes
    import ctypes as C
    m = d2.UnitCubeMesh(1, 1, 1)
    V = d2.FunctionSpace(m, "Lagrange", 1)
    P = V.pattern()
    lib = _capi.lib()
    f = _capi.make_form(_capi.FORM_FUNCTIONAL, _capi.COEFF_CONSTANT, (1.0,))
    assert lib.db2_assemble_scalar(None, C.byref(f), None, None, None) == 1
    assert lib.db2_assemble_scalar(m.handle, C.byref(f), None, None, None) == 1  # out NULL
    assert lib.db2_assemble_local(V.handle, None, None, None, None, 1, None, None, None) == 1
    assert lib.db2_assemble_facets_bc(P.handle, None, None, None, None, None, None, None, None, None) == 1
    assert lib.db2_vector_write_xml(b"/nonexistent_dir/x.xml", 3, None) == 1
    n = C.c_int64(0)
    assert lib.db2_vector_read_xml(b"/nonexistent_dir/x.xml", C.byref(n), None) == 1
    assert lib.db2_mesh_write_xml(None, b"x.xml") == 1
    with pytest.raises(NotImplementedError):
        d2.assemble(d2.inner(d2.grad(d2.TrialFunction(V)), d2.grad(d2.TestFunction(V))) * d2.ds)
    with pytest.raises(NotImplementedError):
        d2.assemble_action(d2.TrialFunction(V) * d2.TestFunction(V) * d2.ds, d2.Vector.__new__(d2.Vector))



def test_row_range_tiles_cover_exactly_the_range():
    """A rank's row range (row-partitioned assembly): the tiles cover exactly
    the nodes [begin, end), for every component, with no overlap."""
    m = d2.UnitCubeMesh(3, 3, 3)
    V = d2.VectorFunctionSpace(m, "Lagrange", 2)
    P = V.pattern()
    nn = V.dim() // 3
    for a, b in [(0, nn), (5, 77), (0, 0), (nn - 3, nn), (m.num_vertices() - 2, m.num_vertices() + 9)]:
        P.set_row_range(a, b)
        t = P.plan()["tiles"]
        for c in range(3):
            tc = t[t[:, 0] == c]
            covered = np.concatenate([np.arange(n0, n1) for _, n0, n1, _ in tc]) if len(tc) else np.array([], int)
            assert np.array_equal(np.sort(covered), np.arange(a, b))
    P.set_row_range(0, nn)
    assert len(P.plan()["tiles"]) > 0
    for a, b in [(-1, 3), (5, 4), (0, nn + 1)]:
        with pytest.raises(_capi.DB2Error):
            P.set_row_range(a, b)


def test_misaligned_output_arrays_are_refused_on_the_host():
    """The assembly writes its CSR values with 16-byte bulk copies from an
    8-byte-aligned base: an output pointer that is not 8-byte aligned is an
    argument error raised before any device work (no GPU needed here)."""
    import ctypes as C
    V = d2.FunctionSpace(d2.UnitSquareMesh(2, 2), "Lagrange", 1)
    a = _capi.make_form(_capi.FORM_DIFFUSION, _capi.COEFF_NONE, (1.0,))
    with pytest.raises(_capi.DB2Error, match="8-byte aligned"):
        _capi.call("db2_assemble_matrix", V.pattern().handle, C.byref(a), None, _capi.FP64,
                   C.c_void_p(0x1004), 0, None)
