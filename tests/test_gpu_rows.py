"""Row-partitioned assembly (one rank's share of a single mesh): assembling
the node-row ranges of shard.row_partition one after another into the same
arrays reproduces the full assembly bit for bit -- each rank computes its
rows completely from the cells around them, so ranks exchange nothing."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import dolfin_b200 as d2
from dolfin_b200 import shard, synthetic


def _problem(kind):
    n = 5
    mesh = d2.UnitCubeMesh(n, n, n)
    mesh.set_coordinates(synthetic.jitter_interior(mesh.coordinates(), n, 0.15, 21))
    bcs = None
    if kind == "elas":
        V = d2.VectorFunctionSpace(mesh, "Lagrange", 2)
        u, v = d2.TrialFunction(V), d2.TestFunction(V)
        eps = lambda w: d2.sym(d2.grad(w))
        a = d2.inner(2 * d2.Constant(0.4) * eps(u) + d2.Constant(0.6) * d2.tr(eps(u)) * d2.Identity(3),
                     eps(v)) * d2.dx
        L = d2.inner(d2.Constant((0.0, 0.0, -1.0)), v) * d2.dx
    else:
        deg = 2 if kind.startswith("p2") else 1
        V = d2.FunctionSpace(mesh, "Lagrange", deg)
        W = d2.FunctionSpace(mesh, "Lagrange", 1)
        kappa = d2.Function(W, synthetic.uniform_field(mesh.num_vertices(), 0.5, 2.0, 22))
        f = d2.Function(W, synthetic.uniform_field(mesh.num_vertices(), -1.0, 1.0, 23))
        u, v = d2.TrialFunction(V), d2.TestFunction(V)
        a = kappa * d2.inner(d2.grad(u), d2.grad(v)) * d2.dx
        L = f * v * d2.dx
        if "ds" in kind:
            # exterior-facet terms: boundary mass and a P1 Neumann load
            a = a + d2.Constant(0.5) * u * v * d2.ds
            L = L + kappa * v * d2.ds
        if kind.endswith("bc"):
            where = "on_boundary" if "ds" not in kind else (lambda x, on: on and x[0] < 1e-12)
            bcs = d2.DirichletBC(V, 0.25, where)
    return V, a, L, bcs


@pytest.mark.parametrize("kind", ["p2", "elas", "p1bc", "p2bc", "p1ds", "p2ds", "p1dsbc"])
@pytest.mark.parametrize("nranks", [2, 3])
def test_row_partitioned_assembly_equals_full(kind, nranks):
    V, a, L, bcs = _problem(kind)
    S = d2.SystemAssembler(a, L, bcs)
    A, b = S.assemble()
    ref_vals, ref_b = A.values_tensor().clone(), b.tensor().clone()
    P = A.pattern
    nn = V.dim() // V.value_size()
    cuts = shard.row_partition(P.plan()["inc_ptr"], nranks)
    A2, b2 = d2.Matrix(), d2.Vector(n=V.dim())
    A2.init(P)
    A2.values_tensor().fill_(float("nan"))  # every entry must be written by some rank
    b2.tensor().fill_(float("nan"))
    try:
        for r in range(nranks):
            P.set_row_range(int(cuts[r]), int(cuts[r + 1]))
            S.assemble(A2, b2)
    finally:
        P.set_row_range(0, nn)
    torch.cuda.synchronize()
    assert torch.equal(A2.values_tensor(), ref_vals)
    assert torch.equal(b2.tensor(), ref_b)


@pytest.mark.parametrize("kind", ["p2", "elas", "p1bc", "p1ds", "p1dsbc"])
@pytest.mark.parametrize("nranks", [2, 3])
def test_row_blocks_held_alone_equal_full(kind, nranks):
    """Each rank holds only its row block (shard.RowBlock: its CSR rows and b
    entries, allocated alone); placed back at their global rows, the blocks
    are the full assembly bit for bit."""
    V, a, L, bcs = _problem(kind)
    A, b = d2.SystemAssembler(a, L, bcs).assemble()
    ref_vals, ref_b = A.values_tensor().cpu().numpy(), b.get_local()
    P = A.pattern
    frp, _ = P.csr_host()
    nn = V.dim() // V.value_size()
    cuts = shard.row_partition(P.plan()["inc_ptr"], nranks)
    vals = np.full(len(ref_vals), np.nan)
    bv = np.full(len(ref_b), np.nan)
    try:
        for r in range(nranks):
            blk = shard.RowBlock(V, int(cuts[r]), int(cuts[r + 1]))
            assert blk.vals.numel() < len(ref_vals) or nranks == 1
            bvals, bb = blk.assemble_system(a, L, bcs)
            torch.cuda.synchronize()
            rp, _ = blk.csr_host()
            bvals, bb = bvals.cpu().numpy(), bb.cpu().numpy()
            for i, dof in enumerate(blk.dofs()):
                vals[frp[dof]:frp[dof + 1]] = bvals[rp[i]:rp[i + 1]]
            bv[blk.dofs()] = bb
    finally:
        P.set_row_range(0, nn)
    assert np.array_equal(vals, ref_vals)
    assert np.array_equal(bv, ref_b)
    with pytest.raises(RuntimeError):
        P.set_row_block(0, nn // 2)
        try:
            d2.SystemAssembler(a, L, bcs).assemble(A, b)
        finally:
            P.set_row_range(0, nn)


@pytest.mark.parametrize("kind", ["p2", "elas", "p2bc"])
def test_fp32_row_blocks_equal_fp32_full(kind):
    """The FP32-contraction path (FP32 row segments, converted on the way
    out) through row-block storage: the blocks placed back at their global
    rows equal the FP32 whole-matrix assembly bit for bit."""
    V, a, L, bcs = _problem(kind)
    A, b = d2.SystemAssembler(a, L, bcs, "fp32").assemble()
    ref_vals, ref_b = A.values_tensor().cpu().numpy(), b.get_local()
    P = A.pattern
    frp, _ = P.csr_host()
    nn = V.dim() // V.value_size()
    cuts = shard.row_partition(P.plan()["inc_ptr"], 3)
    vals = np.full(len(ref_vals), np.nan)
    bv = np.full(len(ref_b), np.nan)
    try:
        for r in range(3):
            blk = shard.RowBlock(V, int(cuts[r]), int(cuts[r + 1]))
            bvals, bb = blk.assemble_system(a, L, bcs, precision="fp32")
            torch.cuda.synchronize()
            rp, _ = blk.csr_host()
            bvals, bb = bvals.cpu().numpy(), bb.cpu().numpy()
            for i, dof in enumerate(blk.dofs()):
                vals[frp[dof]:frp[dof + 1]] = bvals[rp[i]:rp[i + 1]]
            bv[blk.dofs()] = bb
    finally:
        P.set_row_range(0, nn)
    assert np.array_equal(vals, ref_vals)
    assert np.array_equal(bv, ref_b)
