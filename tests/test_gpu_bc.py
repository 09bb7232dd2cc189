"""SystemAssembler with DirichletBC on the GPU: the reference's known answer
and the oracle's SystemAssembler::apply_bc restatement on jittered meshes."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import dolfin_b200 as d2
from dolfin_b200 import synthetic


def test_cell_assembly_bc_known_answer():
    # python/test/unit/fem/test_system_assembler.py:54-90
    mesh = d2.UnitCubeMesh(4, 4, 4)
    V = d2.FunctionSpace(mesh, "Lagrange", 1)
    bc = d2.DirichletBC(V, 1.0, "on_boundary")
    u, v = d2.TrialFunction(V), d2.TestFunction(V)
    f = d2.Constant(10)
    a = d2.inner(d2.grad(u), d2.grad(v)) * d2.dx
    L = d2.inner(f, v) * d2.dx
    A, b = d2.assemble_system(a, L, bc)
    assert round(A.norm("frobenius") - 96.847818767384, 10) == 0
    assert round(b.norm("l2") - 96.564760289080, 10) == 0
    S = d2.SystemAssembler(a, L, bc)
    A2, b2 = S.assemble(d2.Matrix(), d2.Vector(n=V.dim()))
    assert round(A2.norm("frobenius") - 96.847818767384, 10) == 0
    assert round(b2.norm("l2") - 96.564760289080, 10) == 0


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-12), ("fp32", 1e-6)])
@pytest.mark.parametrize("deg,vs", [(2, 1), (1, 3), (2, 3)])
def test_bc_against_oracle(orc, deg, vs, precision, tol):
    """FP64, and the FP32-contraction path (FP32 element rows and row
    segments; the Dirichlet columns move to b from the FP32 rows)."""
    n = 3
    mesh = d2.UnitCubeMesh(n, n, n)
    om = orc.unit_cube_mesh(n, n, n)
    x = synthetic.jitter_interior(om.coords, n, 0.1, 3)
    mesh.set_coordinates(x)
    om.coords = x
    V = d2.FunctionSpace(mesh, "Lagrange", deg, value_size=vs)
    u, v = d2.TrialFunction(V), d2.TestFunction(V)
    left = lambda p, on_b: on_b and p[0] < 1e-12
    if vs == 1:
        W = d2.FunctionSpace(mesh, "Lagrange", 1)
        kv = synthetic.uniform_field(om.nv, 0.5, 2.0, 4)
        a = d2.Function(W, kv) * d2.inner(d2.grad(u), d2.grad(v)) * d2.dx
        L = d2.Constant(3.0) * v * d2.dx
        bc = d2.DirichletBC(V, lambda p: 1.0 + p[1] * p[2], "on_boundary")
        fa = orc.form(orc.DIFFUSION, 3, deg, 1, coeff=orc.COEFF_P1)
        fL = orc.form(orc.LOAD, 3, deg, 1, coeff=orc.COEFF_CONST, c=(3.0,))
        wa = kv
    else:
        mu, lm = 0.7, 1.3
        eps = lambda w: d2.sym(d2.grad(w))
        a = d2.inner(2 * d2.Constant(mu) * eps(u) + d2.Constant(lm) * d2.tr(eps(u)) * d2.Identity(3), eps(v)) * d2.dx
        L = d2.inner(d2.Constant((0.0, 0.5, -1.0)), v) * d2.dx
        bc = d2.DirichletBC(V, (0.1, 0.0, -0.2), left)
        fa = orc.form(orc.ELASTICITY, 3, deg, 3, mu=mu, lmbda=lm)
        fL = orc.form(orc.LOAD, 3, deg, 3, coeff=orc.COEFF_CONST, c=(0.0, 0.5, -1.0))
        wa = None
    A, b = d2.assemble_system(a, L, bc, precision=precision)
    rp, cols, vals = A.data()
    od, N = orc.dofmap(om, deg, vs)
    dofs, bvals = bc.dofs_and_values()
    order = np.argsort(dofs)
    ref, bref = orc.assemble_system(fa, fL, om, od, N, rp, cols, dofs[order].astype(np.int32),
                                    bvals[order], wa=wa)
    scale = np.repeat(np.maximum.reduceat(np.abs(ref), rp[:-1]), np.diff(rp))
    assert np.max(np.abs(vals - ref) / scale) <= tol
    got = b.get_local()
    assert np.max(np.abs(got - bref)) / np.max(np.abs(bref)) <= tol
