"""Assembly on reordered spaces (reorder_dofs_serial = True) against the
oracle assembling directly with the reordered dofmap."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import dolfin_b200 as d2
from dolfin_b200 import synthetic

TOL = 1e-12


@pytest.fixture
def reordered():
    old = d2.parameters["reorder_dofs_serial"]
    d2.parameters["reorder_dofs_serial"] = True
    yield
    d2.parameters["reorder_dofs_serial"] = old


def _row_err(rp, vals, ref):
    scale = np.repeat(np.maximum.reduceat(np.abs(ref), rp[:-1]), np.diff(rp))
    scale[scale == 0] = 1.0
    return float(np.max(np.abs(vals - ref) / scale))


def _vec_err(b, ref):
    return float(np.max(np.abs(b - ref)) / max(np.max(np.abs(ref)), 1e-300))


def _case(orc, tdim, n, seed=31):
    mesh = d2.UnitCubeMesh(n, n, n) if tdim == 3 else d2.UnitSquareMesh(n, n)
    om = orc.unit_cube_mesh(n, n, n) if tdim == 3 else orc.unit_square_mesh(n, n)
    x = synthetic.jitter_interior(om.coords, n, 0.1, seed)
    mesh.set_coordinates(x)
    om.coords = x
    return mesh, om


def _p1_function(W, kv):
    """Function on a (possibly reordered) P1 space with vertex values kv."""
    vals = np.empty_like(kv)
    vals[W.node_numbers()] = kv
    return d2.Function(W, vals)


@pytest.mark.parametrize("tdim,deg", [(2, 2), (3, 1), (3, 2)])
def test_reordered_poisson_system_with_bcs(orc, reordered, tdim, deg):
    mesh, om = _case(orc, tdim, 3 if tdim == 3 else 6)
    V = d2.FunctionSpace(mesh, "Lagrange", deg)
    W = d2.FunctionSpace(mesh, "Lagrange", 1)
    u, v = d2.TrialFunction(V), d2.TestFunction(V)
    kv = synthetic.uniform_field(om.nv, 0.5, 2.0, 32)
    fv = synthetic.uniform_field(om.nv, -1.0, 1.0, 33)
    kappa, f = _p1_function(W, kv), _p1_function(W, fv)
    a = kappa * d2.inner(d2.grad(u), d2.grad(v)) * d2.dx
    L = f * v * d2.dx
    od, N, _ = orc.dofmap_reordered(om, deg)
    # plain assembly
    A = d2.assemble(a)
    rp, cols, vals = A.data()
    orp, ocols = orc.sparsity(N, N, od, od)
    assert np.array_equal(rp, orp) and np.array_equal(cols, ocols)
    fa = orc.form(orc.DIFFUSION, tdim, deg, coeff=orc.COEFF_P1)
    fl = orc.form(orc.LOAD, tdim, deg, coeff=orc.COEFF_P1)
    ref = orc.assemble_matrix(fa, om, od, od, rp, cols, w=kv)
    assert _row_err(rp, vals, ref) <= TOL
    b = d2.assemble(L).get_local()
    assert _vec_err(b, orc.assemble_vector(fl, om, od, N, w=fv)) <= TOL
    # system with a Dirichlet condition on part of the boundary
    bc = d2.DirichletBC(V, lambda p: 1.0 + p[1], lambda p, on_b: on_b and p[0] < 1e-12)
    A2, b2 = d2.assemble_system(a, L, bc)
    dofs, bvals = bc.dofs_and_values()
    order = np.argsort(dofs)
    ref2, bref2 = orc.assemble_system(fa, fl, om, od, N, rp, cols, dofs[order].astype(np.int32),
                                      bvals[order], wa=kv, wL=fv)
    assert _row_err(rp, A2.data()[2], ref2) <= TOL
    assert _vec_err(b2.get_local(), bref2) <= TOL


@pytest.mark.parametrize("deg", [1, 2])
def test_reordered_elasticity_and_traction(orc, reordered, deg):
    mesh, om = _case(orc, 3, 2)
    V = d2.VectorFunctionSpace(mesh, "Lagrange", deg)
    u, v = d2.TrialFunction(V), d2.TestFunction(V)
    mu, lm = 0.6, 1.1
    eps = lambda w: d2.sym(d2.grad(w))
    a = d2.inner(2 * d2.Constant(mu) * eps(u) + d2.Constant(lm) * d2.tr(eps(u)) * d2.Identity(3), eps(v)) * d2.dx
    L = d2.inner(d2.Constant((0.0, 0.5, -1.0)), v) * d2.dx + d2.inner(d2.Constant((1.0, 0.0, 0.0)), v) * d2.ds
    A = d2.assemble(a)
    b = d2.assemble(L).get_local()
    rp, cols, vals = A.data()
    od, N, _ = orc.dofmap_reordered(om, deg, 3)
    ref = orc.assemble_matrix(orc.form(orc.ELASTICITY, 3, deg, 3, mu=mu, lmbda=lm), om, od, od, rp, cols)
    assert _row_err(rp, vals, ref) <= TOL
    bref = orc.assemble_vector(orc.form(orc.LOAD, 3, deg, 3, coeff=orc.COEFF_CONST, c=(0.0, 0.5, -1.0)), om, od, N)
    bref += orc.assemble_vector(orc.form(orc.FACET_LOAD, 3, deg, 3, coeff=orc.COEFF_CONST, c=(1.0, 0.0, 0.0)), om, od, N)
    assert _vec_err(b, bref) <= TOL


def test_reordered_action_adjoint_and_facets(orc, reordered):
    from dolfin_b200.autodiff import vjp_kappa
    mesh, om = _case(orc, 3, 3)
    V = d2.FunctionSpace(mesh, "Lagrange", 2)
    W = d2.FunctionSpace(mesh, "Lagrange", 1)
    u, v = d2.TrialFunction(V), d2.TestFunction(V)
    kv = synthetic.lognormal_field(om.nv, 0.5, 34)
    kappa = _p1_function(W, kv)
    a = kappa * d2.inner(d2.grad(u), d2.grad(v)) * d2.dx
    A = d2.assemble(a)
    x = torch.randn(V.dim(), dtype=torch.float64, device="cuda", generator=torch.Generator("cuda").manual_seed(35))
    y = d2.assemble_action(a, d2.Vector(x)).get_local()
    yref = A.sparray() @ x.cpu().numpy()
    assert _vec_err(y, yref) <= 1e-11
    # adjoint: gA in the reordered CSR order, dkappa by vertex
    rp, cols = V.pattern().csr_host()
    gA = np.random.default_rng(36).standard_normal(cols.shape[0])
    dk = vjp_kappa(V, torch.as_tensor(kv, device="cuda"), torch.as_tensor(gA, device="cuda"))
    od, N, _ = orc.dofmap_reordered(om, 2)
    ref = orc.vjp_diffusion(orc.form(orc.DIFFUSION, 3, 2, 1, coeff=2), om, od, rp, cols, gA)
    assert _vec_err(dk.cpu().numpy(), ref) <= TOL
    # exterior facets
    M = d2.assemble(2.0 * u * v * d2.ds)
    refm = orc.assemble_matrix(orc.form(orc.FACET_MASS, 3, 2, coeff=orc.COEFF_CONST, c=(2.0,)), om, od, od, rp, cols)
    assert _row_err(rp, M.data()[2], refm) <= TOL


def test_reordered_fp32_paths(orc, reordered):
    """The FP32-contraction assembly and both FP32 matrix-free actions (FP32
    quadrature, tensor cores) on a reordered space, against the FP64 results
    there: 1e-6 of the row scale (|A| |x| for the actions)."""
    mesh, om = _case(orc, 3, 4)
    V = d2.FunctionSpace(mesh, "Lagrange", 2)
    W = d2.FunctionSpace(mesh, "Lagrange", 1)
    u, v = d2.TrialFunction(V), d2.TestFunction(V)
    kappa = _p1_function(W, synthetic.lognormal_field(om.nv, 0.5, 37))
    a = kappa * d2.inner(d2.grad(u), d2.grad(v)) * d2.dx
    A = d2.assemble(a)
    rp, cols, vals = A.data()
    A32 = d2.assemble(a, precision="fp32")
    assert _row_err(rp, A32.data()[2], vals) <= 1e-6
    x = torch.randn(V.dim(), dtype=torch.float64, device="cuda", generator=torch.Generator("cuda").manual_seed(38))
    S = A.sparray()
    xn = x.cpu().numpy()
    yref = S @ xn
    mag = abs(S) @ np.abs(xn)
    for prec in ("fp32", "fp32_tc"):
        y = d2.assemble_action(a, d2.Vector(x), precision=prec).get_local()
        assert float(np.max(np.abs(y - yref) / mag)) <= 1e-6, prec
