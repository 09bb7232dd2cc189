"""Meshes whose vertex numbering is spread out: cells whose vertex ids lie
more than 32767 apart (a user mesh with unordered numbering, read from a
DOLFIN XML file; UnitCubeMesh(200), whose cells span 40,603 ids).  Their
incidence records cannot hold every vertex as a 16-bit offset; those
records are marked and the kernel reads the cell's vertices instead.  The
results must still equal the oracle's: pattern bit-exact, FP64 values
within 1e-12 row-scaled."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import dolfin_b200 as d2
from dolfin_b200 import synthetic

FP64_TOL = 1e-12


def row_scaled_err(rp, vals, ref):
    rowmax = np.maximum.reduceat(np.abs(ref), rp[:-1].astype(np.int64))
    rowmax[rowmax == 0] = 1.0
    return float(np.max(np.abs(vals - ref) / np.repeat(rowmax, np.diff(rp))))


def _permuted_mesh(orc, n, seed):
    """UnitCubeMesh(n) jittered, vertices renumbered by a random permutation
    (cell vertex lists re-sorted: an ordered mesh, as MeshEditor::close
    leaves it)."""
    om = orc.unit_cube_mesh(n, n, n)
    x = synthetic.jitter_interior(om.coords, n, 0.15, seed)
    perm = np.random.default_rng(seed + 1).permutation(om.nv)
    xp = np.empty_like(x)
    xp[perm] = x
    cells = np.sort(perm[om.cells.astype(np.int64)], axis=1).astype(np.uint32)
    spread = int(np.max(cells[:, -1].astype(np.int64) - cells[:, 0]))
    return orc.Mesh(3, xp, cells), spread


@pytest.mark.parametrize("deg", [1, 2])
def test_permuted_xml_mesh_poisson(orc, tmp_path, deg):
    om, spread = _permuted_mesh(orc, 34, 70)
    assert spread > 32767 and om.nv > 32768
    path = str(tmp_path / "permuted.xml")
    d2.File(path) << d2.Mesh(om.coords, om.cells)
    mesh = d2.Mesh(path)
    assert np.array_equal(mesh.cells(), om.cells) and np.array_equal(mesh.coordinates(), om.coords)
    V = d2.FunctionSpace(mesh, "Lagrange", deg)
    W = d2.FunctionSpace(mesh, "Lagrange", 1)
    kv = synthetic.uniform_field(om.nv, 0.5, 2.0, 71)
    fv = synthetic.uniform_field(om.nv, -1.0, 1.0, 72)
    kappa, f = d2.Function(W, kv), d2.Function(W, fv)
    u, v = d2.TrialFunction(V), d2.TestFunction(V)
    A, b = d2.assemble_system(kappa * d2.inner(d2.grad(u), d2.grad(v)) * d2.dx, f * v * d2.dx)
    rp, cols, vals = A.data()
    od, N = orc.dofmap(om, deg, 1)
    assert np.array_equal(V.dofmap().cell_dofs_all(), od)
    orp, ocols = orc.sparsity(N, N, od, od)
    assert np.array_equal(rp, orp) and np.array_equal(cols, ocols)
    ref = orc.assemble_matrix(orc.form(orc.DIFFUSION, 3, deg, 1, coeff=orc.COEFF_P1), om, od, od,
                              orp, ocols, w=kv)
    bref = orc.assemble_vector(orc.form(orc.LOAD, 3, deg, 1, coeff=orc.COEFF_P1), om, od, N, w=fv)
    assert row_scaled_err(rp, vals, ref) <= FP64_TOL
    assert float(np.max(np.abs(b.get_local() - bref)) / np.max(np.abs(bref))) <= FP64_TOL
    # the FP32-contraction kernels take the same path
    A32 = d2.assemble(kappa * d2.inner(d2.grad(u), d2.grad(v)) * d2.dx, precision="fp32")
    assert row_scaled_err(rp, A32.values_tensor().cpu().numpy(), ref) <= 1e-6


def test_permuted_mesh_elasticity(orc):
    from oracle import parallel
    om, spread = _permuted_mesh(orc, 32, 80)
    assert spread > 32767
    mesh = d2.Mesh(om.coords, om.cells)
    V = d2.VectorFunctionSpace(mesh, "Lagrange", 2)
    u, v = d2.TrialFunction(V), d2.TestFunction(V)
    mu, lm = 0.4, 0.7
    eps = lambda w: d2.sym(d2.grad(w))
    a = d2.inner(2 * d2.Constant(mu) * eps(u) + d2.Constant(lm) * d2.tr(eps(u)) * d2.Identity(3), eps(v)) * d2.dx
    L = d2.inner(d2.Constant((0.0, 0.0, -1.0)), v) * d2.dx
    A, b = d2.assemble_system(a, L)
    rp, cols, vals = A.data()
    od, N = orc.dofmap(om, 2, 3)
    ocols, ovals, ob, bad, _ = parallel.assemble_rows(
        om, od, N, 3, 10, rp,
        a=dict(kind=orc.ELASTICITY, tdim=3, degree0=2, vsize0=3, mu=mu, lmbda=lm),
        L=dict(kind=orc.LOAD, tdim=3, degree0=2, vsize0=3, coeff=orc.COEFF_CONST, c=(0.0, 0.0, -1.0)),
        nvert=om.nv)
    assert bad == 0 and np.array_equal(cols, ocols)
    assert row_scaled_err(rp, vals, ovals) <= FP64_TOL
    assert float(np.max(np.abs(b.get_local() - ob)) / np.max(np.abs(ob))) <= FP64_TOL


def test_unit_cube_200_p1(orc):
    """UnitCubeMesh(200): 48,000,000 cells, 8,120,601 vertices; a cell's
    vertex ids span up to (n+1)^2 + (n+1) + 1 = 40,603."""
    from oracle import parallel
    n = 200
    mesh = d2.UnitCubeMesh(n, n, n)
    om = orc.unit_cube_mesh(n, n, n)
    V = d2.FunctionSpace(mesh, "Lagrange", 1)
    W = d2.FunctionSpace(mesh, "Lagrange", 1)
    kv = synthetic.uniform_field(om.nv, 0.5, 2.0, 90)
    fv = synthetic.uniform_field(om.nv, -1.0, 1.0, 91)
    kappa, f = d2.Function(W, kv), d2.Function(W, fv)
    u, v = d2.TrialFunction(V), d2.TestFunction(V)
    A, b = d2.assemble_system(kappa * d2.inner(d2.grad(u), d2.grad(v)) * d2.dx, f * v * d2.dx)
    rp, cols, vals = A.data()
    assert len(cols) == 15 * n**3 + 21 * n**2 + 9 * n + 1
    od, N = orc.dofmap(om, 1, 1)
    ocols, ovals, ob, bad, _ = parallel.assemble_rows(
        om, od, N, 1, 4, rp,
        a=dict(kind=orc.DIFFUSION, tdim=3, degree0=1, coeff=orc.COEFF_P1),
        L=dict(kind=orc.LOAD, tdim=3, degree0=1, coeff=orc.COEFF_P1), wa=kv, wL=fv)
    assert bad == 0 and np.array_equal(cols, ocols)
    assert row_scaled_err(rp, vals, ovals) <= FP64_TOL
    assert float(np.max(np.abs(b.get_local() - ob)) / np.max(np.abs(ob))) <= FP64_TOL
