"""Exterior-facet integrals (ds) and functionals on the GPU against the
oracle's restatement of Assembler::assemble_exterior_facets and
SystemAssembler's facet terms; the reference's known answers for
assemble(1*ds) and assemble(1*dx)."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import dolfin_b200 as d2
from dolfin_b200 import synthetic

TOL = 1e-12


def _case(orc, tdim, n, jitter=0.1, seed=5):
    if tdim == 3:
        mesh, om = d2.UnitCubeMesh(n, n, n), orc.unit_cube_mesh(n, n, n)
    else:
        mesh, om = d2.UnitSquareMesh(n, n), orc.unit_square_mesh(n, n)
    if jitter:
        x = synthetic.jitter_interior(om.coords, n, jitter, seed)
        mesh.set_coordinates(x)
        om.coords = x
    return mesh, om


def _row_err(rp, vals, ref):
    scale = np.repeat(np.maximum.reduceat(np.abs(ref), rp[:-1]), np.diff(rp))
    scale[scale == 0] = 1.0
    return float(np.max(np.abs(vals - ref) / scale))


def _vec_err(b, ref):
    return float(np.max(np.abs(b - ref)) / max(np.max(np.abs(ref)), 1e-300))


@pytest.mark.parametrize("mesh_kind,area", [("square", 4.0), ("cube", 6.0)])
def test_functional_known_answers(mesh_kind, area):
    # python/test/unit/fem/test_assembler.py:140-153 (and :431 for x[0])
    mesh = d2.UnitSquareMesh(4, 4) if mesh_kind == "square" else d2.UnitCubeMesh(2, 2, 2)
    assert round(d2.assemble(d2.Constant(1.0) * d2.dx(mesh)) - 1.0, 7) == 0
    assert round(d2.assemble(d2.Constant(1.0) * d2.ds(mesh)) - area, 7) == 0
    x = d2.SpatialCoordinate(mesh)
    assert round(d2.assemble(x[0] * d2.dx(mesh)) - 0.5, 7) == 0


@pytest.mark.parametrize("tdim", [2, 3])
def test_functionals_match_oracle(orc, tdim):
    mesh, om = _case(orc, tdim, 6 if tdim == 3 else 10)
    W = d2.FunctionSpace(mesh, "Lagrange", 1)
    fv = synthetic.uniform_field(om.nv, -1.0, 2.0, seed=6)
    f = d2.Function(W, fv)
    x = d2.SpatialCoordinate(mesh)
    for form, okind, coeff, c, w in [
            (f * d2.dx, orc.FUNCTIONAL, orc.COEFF_P1, (0,), fv),
            (f * d2.ds, orc.FACET_FUNCTIONAL, orc.COEFF_P1, (0,), fv),
            (x[1] * d2.ds(mesh), orc.FACET_FUNCTIONAL, orc.COEFF_X0, (0, 1), None),
            (2.5 * d2.ds(mesh), orc.FACET_FUNCTIONAL, orc.COEFF_CONST, (2.5,), None)]:
        got = d2.assemble(form)
        ref = orc.assemble_scalar(orc.form(okind, tdim, coeff=coeff, c=c), om, w=w)
        assert abs(got - ref) <= TOL * max(abs(ref), 1.0)
        assert d2.assemble(form) == got  # fixed-order reduction: bitwise repeatable


@pytest.mark.parametrize("tdim,deg", [(2, 1), (2, 2), (3, 1), (3, 2)])
@pytest.mark.parametrize("coeff", ["const", "p1"])
def test_facet_load_and_mass(orc, tdim, deg, coeff):
    mesh, om = _case(orc, tdim, 4 if tdim == 3 else 7)
    V = d2.FunctionSpace(mesh, "Lagrange", deg)
    W = d2.FunctionSpace(mesh, "Lagrange", 1)
    u, v = d2.TrialFunction(V), d2.TestFunction(V)
    gv = synthetic.uniform_field(om.nv, 0.5, 2.0, seed=7)
    if coeff == "p1":
        g = d2.Function(W, gv)
        ok = dict(coeff=orc.COEFF_P1)
        w = gv
    else:
        g = d2.Constant(1.75)
        ok = dict(coeff=orc.COEFF_CONST, c=(1.75,))
        w = None
    od, N = orc.dofmap(om, deg)
    b = d2.assemble(g * v * d2.ds).get_local()
    bref = orc.assemble_vector(orc.form(orc.FACET_LOAD, tdim, deg, **ok), om, od, N, w=w)
    assert _vec_err(b, bref) <= TOL
    A = d2.assemble(g * u * v * d2.ds)
    rp, cols, vals = A.data()
    ref = orc.assemble_matrix(orc.form(orc.FACET_MASS, tdim, deg, **ok), om, od, od, rp, cols, w=w)
    assert _row_err(rp, vals, ref) <= TOL


@pytest.mark.parametrize("deg", [1, 2])
def test_vector_traction(orc, deg):
    mesh, om = _case(orc, 3, 3)
    V = d2.VectorFunctionSpace(mesh, "Lagrange", deg)
    v = d2.TestFunction(V)
    t = (0.3, -1.0, 2.0)
    b = d2.assemble(d2.inner(d2.Constant(t), v) * d2.ds).get_local()
    od, N = orc.dofmap(om, deg, 3)
    bref = orc.assemble_vector(orc.form(orc.FACET_LOAD, 3, deg, 3, coeff=orc.COEFF_CONST, c=t),
                               om, od, N)
    assert _vec_err(b, bref) <= TOL


@pytest.mark.parametrize("tdim,deg", [(2, 2), (3, 1), (3, 2)])
def test_cell_plus_facet_forms(orc, tdim, deg):
    # Assembler::assemble: the cell loop, then the exterior-facet loop
    mesh, om = _case(orc, tdim, 3 if tdim == 3 else 6)
    V = d2.FunctionSpace(mesh, "Lagrange", deg)
    W = d2.FunctionSpace(mesh, "Lagrange", 1)
    u, v = d2.TrialFunction(V), d2.TestFunction(V)
    kv = synthetic.uniform_field(om.nv, 0.5, 2.0, seed=8)
    kappa = d2.Function(W, kv)
    A = d2.assemble(kappa * d2.inner(d2.grad(u), d2.grad(v)) * d2.dx + 3.0 * kappa * u * v * d2.ds)
    rp, cols, vals = A.data()
    od, N = orc.dofmap(om, deg)
    ref = orc.assemble_matrix(orc.form(orc.DIFFUSION, tdim, deg, coeff=orc.COEFF_P1), om, od, od,
                              rp, cols, w=kv)
    ref += orc.assemble_matrix(orc.form(orc.FACET_MASS, tdim, deg, coeff=orc.COEFF_P1), om, od, od,
                               rp, cols, w=3.0 * kv)
    assert _row_err(rp, vals, ref) <= TOL


@pytest.mark.parametrize("tdim,deg", [(2, 2), (3, 1), (3, 2)])
def test_system_with_facets_and_bcs(orc, tdim, deg):
    # SystemAssembler: facet terms added to the cell tensor before apply_bc
    mesh, om = _case(orc, tdim, 3 if tdim == 3 else 6)
    V = d2.FunctionSpace(mesh, "Lagrange", deg)
    W = d2.FunctionSpace(mesh, "Lagrange", 1)
    u, v = d2.TrialFunction(V), d2.TestFunction(V)
    kv = synthetic.uniform_field(om.nv, 0.5, 2.0, seed=9)
    gv = synthetic.uniform_field(om.nv, -1.0, 1.0, seed=10)
    kappa, g = d2.Function(W, kv), d2.Function(W, gv)
    a = kappa * d2.inner(d2.grad(u), d2.grad(v)) * d2.dx + 2.0 * u * v * d2.ds
    L = d2.Constant(1.5) * v * d2.dx + g * v * d2.ds
    left = lambda p, on_b: on_b and p[0] < 1e-12
    bc = d2.DirichletBC(V, lambda p: 1.0 + p[1], left)
    A, b = d2.assemble_system(a, L, bc)
    rp, cols, vals = A.data()
    od, N = orc.dofmap(om, deg)
    dofs, bvals = bc.dofs_and_values()
    order = np.argsort(dofs)
    ref, bref = orc.assemble_system_ds(
        orc.form(orc.DIFFUSION, tdim, deg, coeff=orc.COEFF_P1),
        orc.form(orc.LOAD, tdim, deg, coeff=orc.COEFF_CONST, c=(1.5,)), om, od, N, rp, cols,
        dofs[order].astype(np.int32), bvals[order], wa=kv,
        a_ds=orc.form(orc.FACET_MASS, tdim, deg, coeff=orc.COEFF_CONST, c=(2.0,)),
        L_ds=orc.form(orc.FACET_LOAD, tdim, deg, coeff=orc.COEFF_P1), wL_ds=gv)
    assert _row_err(rp, vals, ref) <= TOL
    assert _vec_err(b.get_local(), bref) <= TOL
    # without Dirichlet data: the plain system path
    A2, b2 = d2.assemble_system(a, L)
    ref2, bref2 = orc.assemble_system_ds(
        orc.form(orc.DIFFUSION, tdim, deg, coeff=orc.COEFF_P1),
        orc.form(orc.LOAD, tdim, deg, coeff=orc.COEFF_CONST, c=(1.5,)), om, od, N, rp, cols,
        np.zeros(0, np.int32), np.zeros(0), wa=kv,
        a_ds=orc.form(orc.FACET_MASS, tdim, deg, coeff=orc.COEFF_CONST, c=(2.0,)),
        L_ds=orc.form(orc.FACET_LOAD, tdim, deg, coeff=orc.COEFF_P1), wL_ds=gv)
    assert _row_err(rp, A2.data()[2], ref2) <= TOL
    assert _vec_err(b2.get_local(), bref2) <= TOL
