"""assemble_local on the GPU: the reference's known answer on the reference
tetrahedron, the oracle's element tensors, and consistency with global
assembly (cell and exterior-facet parts)."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import dolfin_b200 as d2
from dolfin_b200 import synthetic

TOL = 1e-12


def test_reference_tetrahedron_known_answer(tmp_path):
    # python/test/unit/fem/test_assembler.py:351-387: P1 stiffness on the
    # reference tetrahedron read from XML
    p = tmp_path / "tetrahedron.xml"
    p.write_text('<?xml version="1.0"?><dolfin><mesh celltype="tetrahedron" dim="3">'
                 '<vertices size="4"><vertex index="0" x="0" y="0" z="0"/>'
                 '<vertex index="1" x="1" y="0" z="0"/><vertex index="2" x="0" y="1" z="0"/>'
                 '<vertex index="3" x="0" y="0" z="1"/></vertices><cells size="1">'
                 '<tetrahedron index="0" v0="0" v1="1" v2="2" v3="3"/></cells></mesh></dolfin>')
    mesh = d2.Mesh(str(p))
    V = d2.FunctionSpace(mesh, "Lagrange", 1)
    u, v = d2.TrialFunction(V), d2.TestFunction(V)
    A = d2.assemble_local(d2.inner(d2.grad(u), d2.grad(v)) * d2.dx, 0)
    A0 = np.array([[1 / 2, -1 / 6, -1 / 6, -1 / 6], [-1 / 6, 1 / 6, 0, 0],
                   [-1 / 6, 0, 1 / 6, 0], [-1 / 6, 0, 0, 1 / 6]])
    assert round(np.linalg.norm(A - A0), 7) == 0


@pytest.mark.parametrize("tdim,deg", [(2, 1), (2, 2), (3, 1), (3, 2)])
def test_local_tensors_match_oracle(orc, tdim, deg):
    n = 3 if tdim == 3 else 5
    mesh = d2.UnitCubeMesh(n, n, n) if tdim == 3 else d2.UnitSquareMesh(n, n)
    x = synthetic.jitter_interior(mesh.coordinates(), n, 0.15, 11)
    mesh.set_coordinates(x)
    V = d2.FunctionSpace(mesh, "Lagrange", deg)
    W = d2.FunctionSpace(mesh, "Lagrange", 1)
    u, v = d2.TrialFunction(V), d2.TestFunction(V)
    kv = synthetic.uniform_field(mesh.num_vertices(), 0.5, 2.0, 12)
    kappa = d2.Function(W, kv)
    cells = np.array([0, 7, mesh.num_cells() - 1, 13])
    A = d2.assemble_local(kappa * d2.inner(d2.grad(u), d2.grad(v)) * d2.dx, cells)
    b = d2.assemble_local(kappa * v * d2.dx, cells)
    conn = mesh.cells()
    fa = orc.form(orc.DIFFUSION, tdim, deg, coeff=orc.COEFF_P1)
    fl = orc.form(orc.LOAD, tdim, deg, coeff=orc.COEFF_P1)
    k = A.shape[1]
    for i, c in enumerate(cells):
        xc = x[conn[c]]
        ref = orc.element_tensor(fa, xc, w=kv[conn[c]], size=k * k).reshape(k, k)
        assert np.max(np.abs(A[i] - ref)) <= TOL * np.max(np.abs(ref))
        refb = orc.element_tensor(fl, xc, w=kv[conn[c]], size=k)
        assert np.max(np.abs(b[i] - refb)) <= TOL * np.max(np.abs(refb))


@pytest.mark.parametrize("deg", [1, 2])
def test_local_elasticity_matches_oracle(orc, deg):
    mesh = d2.UnitCubeMesh(2, 2, 2)
    x = synthetic.jitter_interior(mesh.coordinates(), 2, 0.15, 13)
    mesh.set_coordinates(x)
    V = d2.VectorFunctionSpace(mesh, "Lagrange", deg)
    u, v = d2.TrialFunction(V), d2.TestFunction(V)
    mu, lm = 0.8, 1.7
    eps = lambda w: d2.sym(d2.grad(w))
    a = d2.inner(2 * d2.Constant(mu) * eps(u) + d2.Constant(lm) * d2.tr(eps(u)) * d2.Identity(3), eps(v)) * d2.dx
    cells = np.arange(0, mesh.num_cells(), 5)
    A = d2.assemble_local(a, cells)
    L = d2.assemble_local(d2.inner(d2.Constant((0.5, -1.0, 2.0)), v) * d2.dx, cells)
    conn = mesh.cells()
    fa = orc.form(orc.ELASTICITY, 3, deg, 3, mu=mu, lmbda=lm)
    fl = orc.form(orc.LOAD, 3, deg, 3, coeff=orc.COEFF_CONST, c=(0.5, -1.0, 2.0))
    n = A.shape[1]
    for i, c in enumerate(cells):
        ref = orc.element_tensor(fa, x[conn[c]], size=n * n).reshape(n, n)
        assert np.max(np.abs(A[i] - ref)) <= TOL * np.max(np.abs(ref))
        refl = orc.element_tensor(fl, x[conn[c]], size=n)
        assert np.max(np.abs(L[i] - refl)) <= TOL * np.max(np.abs(refl))


@pytest.mark.parametrize("tdim,deg", [(2, 2), (3, 1), (3, 2)])
def test_local_tensors_sum_to_global_assembly(tdim, deg):
    # scatter of every cell's local tensor (dx + ds parts) == assemble(form)
    n = 3 if tdim == 3 else 4
    mesh = d2.UnitCubeMesh(n, n, n) if tdim == 3 else d2.UnitSquareMesh(n, n)
    V = d2.FunctionSpace(mesh, "Lagrange", deg)
    W = d2.FunctionSpace(mesh, "Lagrange", 1)
    u, v = d2.TrialFunction(V), d2.TestFunction(V)
    kv = synthetic.uniform_field(mesh.num_vertices(), 0.5, 2.0, 14)
    kappa = d2.Function(W, kv)
    a = kappa * d2.inner(d2.grad(u), d2.grad(v)) * d2.dx + 2.0 * kappa * u * v * d2.ds
    L = d2.Constant(0.5) * v * d2.dx + kappa * v * d2.ds
    cells = np.arange(mesh.num_cells())
    Ae = d2.assemble_local(a, cells)
    be = d2.assemble_local(L, cells)
    dofs = np.array([V.dofmap().cell_dofs(c) for c in cells])
    N = V.dim()
    Ad = np.zeros((N, N))
    bd = np.zeros(N)
    for c in cells:
        Ad[np.ix_(dofs[c], dofs[c])] += Ae[c]
        bd[dofs[c]] += be[c]
    A = d2.assemble(a).sparray().toarray()
    b = d2.assemble(L).get_local()
    assert np.max(np.abs(Ad - A)) <= 1e-13 * np.max(np.abs(A))
    assert np.max(np.abs(bd - b)) <= 1e-13 * np.max(np.abs(b))
