"""The differentiable assembly (autodiff.AssembleDiffusion, a
torch.autograd.Function) on P1 Poisson, UnitCubeMesh(32): forward A and b
(b = kappa*f*v*dx, the kappa-weighted load) against the oracle, and
gradients from torch.autograd.grad against central differences (h = 1e-6,
64 random directions) of L(kappa) = <gA, A(kappa)> + <gb, b(kappa)>.
Bounds, as |fd - ad| / (|dL/dkappa| |direction|): FP64 <= 1e-8; the
FP32-contraction path (forward and adjoint in FP32 contraction, FP64
geometry and sums) <= 1e-6 against the FP64 differences."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import dolfin_b200 as d2
from dolfin_b200 import synthetic
from dolfin_b200.autodiff import AssembleDiffusion


def _case(n, deg=1):
    mesh = d2.UnitCubeMesh(n, n, n)
    V = d2.FunctionSpace(mesh, "Lagrange", deg)
    nv = mesh.num_vertices()
    kappa = torch.as_tensor(synthetic.lognormal_field(nv, 0.5, 300), device="cuda")
    f = torch.as_tensor(synthetic.uniform_field(nv, -1.0, 1.0, 301), device="cuda")
    return mesh, V, kappa, f


@pytest.mark.parametrize("deg,n", [(1, 32), (2, 6)])
def test_forward_matches_oracle(orc, deg, n):
    mesh, V, kappa, f = _case(n, deg)
    vals, b = AssembleDiffusion.apply(kappa, V, f, True, "fp64")
    om = orc.unit_cube_mesh(n, n, n)
    od, N = orc.dofmap(om, deg, 1)
    rp, cols = V.pattern().csr_host()
    kv, fv = kappa.cpu().numpy(), f.cpu().numpy()
    ref = orc.assemble_matrix(orc.form(orc.DIFFUSION, 3, deg, 1, coeff=orc.COEFF_P1), om, od, od, rp, cols, w=kv)
    bref = orc.assemble_vector(orc.form(orc.LOAD, 3, deg, 1, coeff=orc.COEFF_P1_TIMES_P1), om, od, N, w=kv, w2=fv)
    scale = np.repeat(np.maximum.reduceat(np.abs(ref), rp[:-1]), np.diff(rp))
    assert np.max(np.abs(vals.cpu().numpy() - ref) / scale) <= 1e-12
    assert np.max(np.abs(b.cpu().numpy() - bref)) <= 1e-12 * np.max(np.abs(bref))
    # the same load through the public assemble_system (c*kappa*f*v*dx)
    W = d2.FunctionSpace(mesh, "Lagrange", 1)
    k, fn = d2.Function(W, kappa), d2.Function(W, f)
    u, v = d2.TrialFunction(V), d2.TestFunction(V)
    _, b2 = d2.assemble_system(k * d2.inner(d2.grad(u), d2.grad(v)) * d2.dx, 2.5 * k * fn * v * d2.dx)
    assert np.max(np.abs(b2.get_local() - 2.5 * bref)) <= 1e-12 * np.max(np.abs(2.5 * bref))


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-8), ("fp32", 1e-6)])
def test_autograd_matches_central_differences(precision, tol):
    mesh, V, kappa, f = _case(32)
    g = torch.Generator("cuda").manual_seed(310)
    nnz, N, nv = V.pattern().nnz(), V.dim(), mesh.num_vertices()
    gA = torch.randn(nnz, dtype=torch.float64, device="cuda", generator=g)
    gb = torch.randn(N, dtype=torch.float64, device="cuda", generator=g)
    k = kappa.clone().requires_grad_(True)
    vals, b = AssembleDiffusion.apply(k, V, f, True, precision)
    (dk,) = torch.autograd.grad(torch.dot(gA, vals) + torch.dot(gb, b), k)

    def L(kv):
        with torch.no_grad():
            a, bb = AssembleDiffusion.apply(kv, V, f, True, "fp64")
            return float(torch.dot(gA, a) + torch.dot(gb, bb))

    h = 1e-6
    dirs = torch.randn(64, nv, dtype=torch.float64, device="cuda", generator=g)
    worst = 0.0
    for d in dirs:
        fd = (L(kappa + h * d) - L(kappa - h * d)) / (2 * h)
        ad = float(torch.dot(dk, d))
        worst = max(worst, abs(fd - ad) / (float(dk.norm()) * float(d.norm())))
    assert worst <= tol


def test_unweighted_load_has_no_kappa_gradient_through_b():
    mesh, V, kappa, f = _case(8)
    g = torch.Generator("cuda").manual_seed(320)
    gb = torch.randn(V.dim(), dtype=torch.float64, device="cuda", generator=g)
    k = kappa.clone().requires_grad_(True)
    vals, b = AssembleDiffusion.apply(k, V, f, False, "fp64")
    (dk,) = torch.autograd.grad(torch.dot(gb, b), k, allow_unused=True)
    assert dk is None or float(dk.abs().max()) == 0.0
