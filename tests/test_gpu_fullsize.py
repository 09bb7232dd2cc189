"""Parity at the full benchmark sizes, through size-independent properties
(the oracle covers the same kernels element by element at small sizes):

* stiffness rows sum to zero (constants are in the kernel of grad-grad);
* symmetry, as x^T (A y) = y^T (A x) for random x, y;
* the load vector sums to the integral of its coefficient (sum_i phi_i = 1),
  checked against the engine's own functional;
* the six rigid-body modes are in the kernel of the elasticity matrix;
* two assemblies agree bitwise.

Sizes: P2 Poisson on UnitCubeMesh(96) (204,763,393 nonzeros), vector P2
elasticity on UnitCubeMesh(48) (231,797,385), P1 Poisson on UnitCubeMesh(96).
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = [pytest.mark.gpu,
              pytest.mark.filterwarnings("ignore:Sparse CSR tensor support is in beta")]

import dolfin_b200 as d2
from dolfin_b200 import synthetic


def _matvec(A):
    rp, cols, vals = A.data_device()
    n = rp.numel() - 1
    M = torch.sparse_csr_tensor(rp.long(), cols.long(), vals, size=(n, n))
    return lambda x: (M @ x.unsqueeze(1)).squeeze(1)


def _check_symmetric(mv, n, tol=1e-11):
    g = torch.Generator("cuda").manual_seed(5)
    x = torch.randn(n, dtype=torch.float64, device="cuda", generator=g)
    y = torch.randn(n, dtype=torch.float64, device="cuda", generator=g)
    Ax, Ay = mv(x), mv(y)
    lhs, rhs = float(x @ Ay), float(y @ Ax)
    scale = float(x.norm() * Ay.norm() + y.norm() * Ax.norm())
    assert abs(lhs - rhs) <= tol * scale


@pytest.mark.parametrize("deg,n", [(2, 96), (1, 96)])
def test_poisson_full_size_properties(deg, n):
    mesh = d2.UnitCubeMesh(n, n, n)
    V = d2.FunctionSpace(mesh, "Lagrange", deg)
    W = d2.FunctionSpace(mesh, "Lagrange", 1)
    kappa = d2.Function(W, synthetic.lognormal_field(mesh.num_vertices(), 0.5, 41))
    f = d2.Function(W, synthetic.uniform_field(mesh.num_vertices(), -1.0, 1.0, 42))
    u, v = d2.TrialFunction(V), d2.TestFunction(V)
    a = kappa * d2.inner(d2.grad(u), d2.grad(v)) * d2.dx
    L = f * v * d2.dx
    A, b = d2.assemble_system(a, L)
    vals1 = A.values_tensor().clone()
    b1 = b.tensor().clone()
    d2.assemble_system(a, L, A_tensor=A, b_tensor=b)
    assert torch.equal(vals1, A.values_tensor()) and torch.equal(b1, b.tensor())
    mv = _matvec(A)
    rowsum = mv(torch.ones(V.dim(), dtype=torch.float64, device="cuda"))
    assert float(rowsum.abs().max()) <= 1e-12 * float(A.values_tensor().abs().max()) * 8
    _check_symmetric(mv, V.dim())
    total = float(b.tensor().sum())
    integral = d2.assemble(f * d2.dx)
    assert abs(total - integral) <= 1e-11 * float(b.tensor().abs().sum())


def _node_coordinates(mesh, V):
    """Coordinates of the P2 nodes (vertices, then edge midpoints) of V."""
    x = mesh.coordinates()
    cells = mesh.cells()
    nn = V.dim() // V.value_size()
    cd = V.dofmap().cell_dofs_all()[:, :10]  # component-0 dofs are the node numbers
    X = np.zeros((nn, 3))
    X[:x.shape[0]] = x
    edges = [(2, 3), (1, 3), (1, 2), (0, 3), (0, 2), (0, 1)]
    for e, (p, q) in enumerate(edges):
        X[cd[:, 4 + e]] = 0.5 * (x[cells[:, p]] + x[cells[:, q]])
    return X


def test_elasticity_full_size_rigid_modes():
    n = 48
    mesh = d2.UnitCubeMesh(n, n, n)
    mesh.set_coordinates(synthetic.jitter_interior(mesh.coordinates(), n, 0.15, 43))
    V = d2.VectorFunctionSpace(mesh, "Lagrange", 2)
    u, v = d2.TrialFunction(V), d2.TestFunction(V)
    E, nu = 1.0, 0.3
    mu, lm = d2.Constant(E / (2 * (1 + nu))), d2.Constant(E * nu / ((1 + nu) * (1 - 2 * nu)))
    eps = lambda w: d2.sym(d2.grad(w))
    a = d2.inner(2 * mu * eps(u) + lm * d2.tr(eps(u)) * d2.Identity(3), eps(v)) * d2.dx
    L = d2.inner(d2.Constant((0.0, 0.0, -1.0)), v) * d2.dx
    A, b = d2.assemble_system(a, L)
    vals1 = A.values_tensor().clone()
    d2.assemble_system(a, L, A_tensor=A, b_tensor=b)
    assert torch.equal(vals1, A.values_tensor())
    mv = _matvec(A)
    X = torch.as_tensor(_node_coordinates(mesh, V), device="cuda")
    nn = X.shape[0]
    amax = float(A.values_tensor().abs().max())
    modes = []
    for c in range(3):  # translations (component-major dofs)
        r = torch.zeros(3, nn, dtype=torch.float64, device="cuda")
        r[c] = 1.0
        modes.append(r.reshape(-1))
    for w in torch.eye(3, dtype=torch.float64, device="cuda"):  # rotations w x X
        modes.append(torch.linalg.cross(w.expand_as(X), X).T.reshape(-1))
    for r in modes:
        assert float(mv(r).abs().max()) <= 1e-12 * amax * 8 * float(r.abs().max())
    _check_symmetric(mv, V.dim())
    bz = b.tensor().reshape(3, nn)
    assert abs(float(bz[2].sum()) + 1.0) <= 1e-11 * float(bz[2].abs().sum())
    assert float(bz[:2].abs().max()) == 0.0
