"""Pins the CPU oracle against the reference's own known-answer tests.

Every expected number below is quoted from the reference test-suite
(file:line given per test); tolerances are the reference's own
(``round(x - ref, 10) == 0`` i.e. 1e-10 absolute, unless stated).
"""
from math import factorial

import numpy as np
import pytest


def test_quadrature_exact_monomials(orc):
    # The oracle integrates with a collapsed Gauss--Jacobi rule; it must be
    # exact for the polynomial degree it is asked for.
    for d in (1, 2, 3):
        for deg in range(0, 6):
            for a in range(deg + 1):
                for b in range(deg + 1 - a if d >= 2 else 1):
                    for c in range(deg + 1 - a - b if d >= 3 else 1):
                        exact = factorial(a) * factorial(b) * factorial(c) / factorial(a + b + c + d)
                        assert abs(orc.quadrature_monomial(d, deg, a, b, c) - exact) < 1e-15


def test_reference_assembly_tet(orc):
    # python/test/unit/fem/test_assembler.py:351-387 (test_reference_assembly):
    # P1 stiffness and mass on the reference tetrahedron (tetrahedron.xml).
    xc = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]], float)
    A = orc.element_tensor(orc.form(orc.DIFFUSION, 3), xc, size=16).reshape(4, 4)
    M = orc.element_tensor(orc.form(orc.MASS, 3), xc, size=16).reshape(4, 4)
    A0 = np.array([[1 / 2, -1 / 6, -1 / 6, -1 / 6], [-1 / 6, 1 / 6, 0, 0],
                   [-1 / 6, 0, 1 / 6, 0], [-1 / 6, 0, 0, 1 / 6]])
    M0 = np.full((4, 4), 1 / 120) + np.eye(4) / 120
    assert round(np.linalg.norm(A - A0), 7) == 0
    assert round(np.linalg.norm(M - M0), 7) == 0


def test_cell_assembly_1D(orc):
    # test_assembler.py:39-55: P1 on UnitIntervalMesh(48), f = 10.
    m = orc.unit_interval_mesh(48)
    dofs, n = orc.dofmap(m, 1)
    rp, cols = orc.sparsity(n, n, dofs, dofs)
    A = orc.assemble_matrix(orc.form(orc.DIFFUSION, 1), m, dofs, dofs, rp, cols)
    b = orc.assemble_vector(orc.form(orc.LOAD, 1, coeff=orc.COEFF_CONST, c=(10,)), m, dofs, n)
    assert round(np.linalg.norm(A) - 811.75365721381274397572, 10) == 0
    assert round(np.linalg.norm(b) - 1.43583841167606474087, 10) == 0


def test_cell_assembly_vector_dg1(orc):
    # test_assembler.py:58-77 and test_system_assembler.py:30-51: vector DG1
    # inner(eps(v), eps(u))*dx and inner(v, f)*dx, f = (10, 20, 30), on
    # UnitCubeMesh(4,4,4).  eps:eps == elasticity with mu = 1/2, lambda = 0.
    m = orc.unit_cube_mesh(4, 4, 4)
    dofs, n = orc.dofmap(m, 1, 3, orc.DG)
    rp, cols = orc.sparsity(n, n, dofs, dofs)
    a = orc.form(orc.ELASTICITY, 3, 1, 3, family0=orc.DG, family1=orc.DG, mu=0.5, lmbda=0.0)
    L = orc.form(orc.LOAD, 3, 1, 3, family0=orc.DG, coeff=orc.COEFF_CONST, c=(10, 20, 30))
    A = orc.assemble_matrix(a, m, dofs, dofs, rp, cols)
    b = orc.assemble_vector(L, m, dofs, n)
    assert round(np.linalg.norm(A) - 4.3969686527582512, 10) == 0
    assert round(np.linalg.norm(b) - 0.95470326978246278, 10) == 0


def test_cell_assembly_bc_system(orc):
    # test_system_assembler.py:54-90 (test_cell_assembly_bc): P1 Poisson on
    # UnitCubeMesh(4,4,4), DirichletBC(V, 1.0, "on_boundary"), f = 10,
    # assemble_system (symmetric application, SystemAssembler::apply_bc).
    m = orc.unit_cube_mesh(4, 4, 4)
    dofs, n = orc.dofmap(m, 1)
    rp, cols = orc.sparsity(n, n, dofs, dofs)
    bc = orc.boundary_vertices(m)
    A, b = orc.assemble_system(orc.form(orc.DIFFUSION, 3),
                               orc.form(orc.LOAD, 3, coeff=orc.COEFF_CONST, c=(10,)),
                               m, dofs, n, rp, cols, bc, np.ones(len(bc)))
    assert round(np.linalg.norm(A) - 96.847818767384, 10) == 0
    assert round(np.linalg.norm(b) - 96.564760289080, 10) == 0


def test_nonsquare_assembly_p2_triangle(orc):
    # test_assembler.py:321-347 (test_nonsquare_assembly): VectorElement P2 x
    # P1 on UnitSquareMesh(16,16); div(v)*p*dx and inner(grad(p), v)*dx.
    m = orc.unit_square_mesh(16, 16)
    d0, n0 = orc.dofmap(m, 2, 2)
    d1, n1 = orc.dofmap(m, 1, 1)
    rp, cols = orc.sparsity(n0, n1, d0, d1)
    A = orc.assemble_matrix(orc.form(orc.DIV_P, 2, 2, 2, 1, 1), m, d0, d1, rp, cols)
    assert round(np.linalg.norm(A) - 9.6420303878382718e-01, 10) == 0
    A = orc.assemble_matrix(orc.form(orc.GRADP_V, 2, 2, 2, 1, 1), m, d0, d1, rp, cols)
    assert round(np.linalg.norm(A) - 0.935414346693, 10) == 0


def test_matrix_nnz_p2_p1(orc):
    # python/test/unit/la/test_matrix.py:60-86,405-407: B = v*s*dx with v P2,
    # s P1 on UnitSquareMesh(21,23): B.nnz() == 9398 and B.size(1) == 528.
    m = orc.unit_square_mesh(21, 23)
    d0, n0 = orc.dofmap(m, 2)
    d1, n1 = orc.dofmap(m, 1)
    rp, cols = orc.sparsity(n0, n1, d0, d1)
    assert cols.shape[0] == 9398
    assert n1 == 528


@pytest.mark.parametrize("n,area", [(2, 1.0), (3, 1.0)])
def test_functional_assembly(orc, n, area):
    # test_assembler.py:144-153 (assemble(1*dx) == 1) and :431 (x[0]*dx == 0.5).
    m = orc.unit_cube_mesh(n, n, n)
    one = orc.assemble_scalar(orc.form(orc.FUNCTIONAL, 3, coeff=orc.COEFF_CONST, c=(1.0,)), m)
    x0 = orc.assemble_scalar(orc.form(orc.FUNCTIONAL, 3, coeff=orc.COEFF_X0), m)
    assert round(one - area, 7) == 0
    assert round(x0 - 0.5, 7) == 0
    m2 = orc.unit_square_mesh(16, 16)
    assert round(orc.assemble_scalar(orc.form(orc.FUNCTIONAL, 2, coeff=orc.COEFF_X0), m2) - 0.5, 7) == 0


@pytest.mark.parametrize("n", [1, 2, 4, 32])
def test_p1_sparsity_count(orc, n):
    # Closed form for the Kuhn (6 tets per cube) mesh: nnz = 15n^3 + 21n^2 + 9n + 1.
    m = orc.unit_cube_mesh(n, n, n)
    d, N = orc.dofmap(m, 1)
    rp, cols = orc.sparsity(N, N, d, d)
    assert cols.shape[0] == 15 * n**3 + 21 * n**2 + 9 * n + 1


@pytest.mark.parametrize("n", [1, 2, 4, 6])
def test_p2_sparsity_count(orc, n):
    # nnz_P2(n) = 230 n^3 + 138 n^2 + 24 n + 1 on the Kuhn mesh.
    m = orc.unit_cube_mesh(n, n, n)
    d, N = orc.dofmap(m, 2)
    assert N == (2 * n + 1) ** 3
    rp, cols = orc.sparsity(N, N, d, d)
    assert cols.shape[0] == 230 * n**3 + 138 * n**2 + 24 * n + 1


def test_box_mesh_ordering(orc):
    # BoxMesh.cpp:109-159: vertices z-y-x lexicographic; 6 tets per cube,
    # each cell's vertices sorted (TetrahedronCell::order).
    m = orc.unit_cube_mesh(2, 3, 4)
    assert m.nv == 3 * 4 * 5 and m.nc == 6 * 24
    assert np.all(np.diff(m.cells.astype(np.int64), axis=1) > 0)
    assert np.allclose(m.coords[1], [0.5, 0, 0]) and np.allclose(m.coords[3], [0, 1 / 3, 0])
    assert m.cells[0].tolist() == [0, 1, 4, 16]


def test_edge_numbering_key_order(orc):
    # TopologyComputation.cpp:152-330: edges numbered in sorted (v0<v1) key order.
    m = orc.unit_cube_mesh(3, 2, 2)
    ce, ev = orc.edges(m)
    keys = ev[:, 0].astype(np.int64) * (1 << 32) + ev[:, 1]
    assert np.all(np.diff(keys) > 0)
    tet = [(2, 3), (1, 3), (1, 2), (0, 3), (0, 2), (0, 1)]
    for c in range(m.nc):
        for e, (p, q) in enumerate(tet):
            assert tuple(ev[ce[c, e]]) == (m.cells[c, p], m.cells[c, q])


@pytest.mark.parametrize("mesh,area", [("square", 4.0), ("cube", 6.0)])
def test_facet_functional_area(orc, mesh, area):
    # python/test/unit/fem/test_assembler.py:140-153: assemble(1*ds(mesh)) is
    # the boundary measure: 4.0 on UnitSquareMesh(4, 4), 6.0 on UnitCubeMesh(2, 2, 2).
    m = orc.unit_square_mesh(4, 4) if mesh == "square" else orc.unit_cube_mesh(2, 2, 2)
    f = orc.form(orc.FACET_FUNCTIONAL, m.tdim, coeff=orc.COEFF_CONST, c=(1.0,))
    assert round(orc.assemble_scalar(f, m) - area, 7) == 0


@pytest.mark.parametrize("tdim,n", [(2, 5), (3, 3)])
def test_exterior_facets(orc, tdim, n):
    # boundary facets of the box mesh: 4n edges (2D), 2 per boundary square (3D);
    # numbered in sorted-key order, each opposite the listed local vertex
    m = orc.unit_square_mesh(n, n) if tdim == 2 else orc.unit_cube_mesh(n, n, n)
    fc, fl = orc.exterior_facets(m)
    assert fc.shape[0] == (4 * n if tdim == 2 else 12 * n * n)
    keys = [tuple(sorted(np.delete(m.cells[c], f).tolist())) for c, f in zip(fc, fl)]
    assert keys == sorted(keys) and len(set(keys)) == len(keys)
    x = m.coords
    for c, f in zip(fc, fl):
        pts = x[np.delete(m.cells[c], f)]
        assert np.any(np.all(np.isclose(pts, 0.0), axis=0) | np.all(np.isclose(pts, 1.0), axis=0))


@pytest.mark.parametrize("deg", [1, 2])
@pytest.mark.parametrize("tdim", [2, 3])
def test_facet_integral_identities(orc, tdim, deg):
    # sum_i int_dO g phi_i = g |dO|;  1^T M_ds 1 = |dO|;  int_dO x_i ds = |dO| / 2
    n = 4 if tdim == 2 else 2
    m = orc.unit_square_mesh(n, n) if tdim == 2 else orc.unit_cube_mesh(n, n, n)
    area = 4.0 if tdim == 2 else 6.0
    d, N = orc.dofmap(m, deg)
    b = orc.assemble_vector(orc.form(orc.FACET_LOAD, tdim, deg, coeff=orc.COEFF_CONST, c=(2.5,)),
                            m, d, N)
    assert abs(b.sum() - 2.5 * area) < 1e-12
    rp, cols = orc.sparsity(N, N, d, d)
    M = orc.assemble_matrix(orc.form(orc.FACET_MASS, tdim, deg), m, d, d, rp, cols)
    assert abs(M.sum() - area) < 1e-12
    for comp in range(tdim):
        fx = orc.form(orc.FACET_FUNCTIONAL, tdim, coeff=orc.COEFF_X0, c=(0.0, comp))
        assert abs(orc.assemble_scalar(fx, m) - area / 2) < 1e-12


def test_system_with_facets_without_bcs(orc):
    # with no Dirichlet dofs the cell-wise system is the sum of the cell and
    # exterior-facet assemblies
    m = orc.unit_cube_mesh(2, 2, 2)
    d, N = orc.dofmap(m, 2)
    rp, cols = orc.sparsity(N, N, d, d)
    kv = np.linspace(0.5, 2.0, m.nv)
    a = orc.form(orc.DIFFUSION, 3, 2, coeff=orc.COEFF_P1)
    a_ds = orc.form(orc.FACET_MASS, 3, 2, coeff=orc.COEFF_CONST, c=(3.0,))
    L = orc.form(orc.LOAD, 3, 2, coeff=orc.COEFF_CONST, c=(1.0,))
    L_ds = orc.form(orc.FACET_LOAD, 3, 2, coeff=orc.COEFF_P1)
    vals, b = orc.assemble_system_ds(a, L, m, d, N, rp, cols, np.zeros(0, np.int32), np.zeros(0),
                                     wa=kv, a_ds=a_ds, L_ds=L_ds, wL_ds=kv)
    A1 = orc.assemble_matrix(a, m, d, d, rp, cols, w=kv) + orc.assemble_matrix(a_ds, m, d, d, rp, cols)
    b1 = orc.assemble_vector(L, m, d, N) + orc.assemble_vector(L_ds, m, d, N, w=kv)
    assert np.max(np.abs(vals - A1)) < 1e-13 * np.max(np.abs(A1))
    assert np.max(np.abs(b - b1)) < 1e-13 * np.max(np.abs(b1))
