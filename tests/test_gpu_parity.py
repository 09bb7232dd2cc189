"""GPU parity: the CUDA engine against the CPU oracle on the same seeded
inputs.  Pattern and dofmap bit-exact; FP64 values within 1e-12 relative
(row-scaled: |A_ij - R_ij| <= 1e-12 * max_j |R_ij|, vectors scaled by
max |b|); the FP32-contraction path within 1e-6 of the FP64 oracle."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import dolfin_b200 as d2
from dolfin_b200 import synthetic

FP64_TOL = 1e-12
FP32_TOL = 1e-6


def row_scaled_err(rp, vals, ref):
    n = rp.shape[0] - 1
    lens = np.diff(rp)
    rowmax = np.maximum.reduceat(np.abs(ref), rp[:-1]) if n else np.zeros(0)
    scale = np.repeat(rowmax, lens)
    scale[scale == 0] = 1.0
    return float(np.max(np.abs(vals - ref) / scale)) if vals.size else 0.0


def vec_err(b, ref):
    return float(np.max(np.abs(b - ref)) / max(np.max(np.abs(ref)), 1e-300))


class Case:
    """Engine mesh + oracle mesh on identical coordinates."""

    def __init__(self, orc, tdim, n, jitter=0.0, seed=0):
        if tdim == 3:
            self.mesh = d2.UnitCubeMesh(n, n, n)
            self.om = orc.unit_cube_mesh(n, n, n)
        else:
            self.mesh = d2.UnitSquareMesh(n, n)
            self.om = orc.unit_square_mesh(n, n)
        if jitter:
            x = synthetic.jitter_interior(self.om.coords, n, jitter, seed)
            self.mesh.set_coordinates(x)
            self.om.coords = x
        self.tdim = tdim


def _oracle_matrix(orc, case, okind, deg, vs, rp, cols, w=None, coeff=0, c=(0, 0, 0), mu=0, lm=0):
    od, N = orc.dofmap(case.om, deg, vs)
    f = orc.form(okind, case.tdim, deg, vs, coeff=coeff, c=c, mu=mu, lmbda=lm)
    return orc.assemble_matrix(f, case.om, od, od, rp, cols, w=w), od, N


@pytest.mark.parametrize("tdim,deg,n", [(3, 1, 6), (3, 2, 3), (2, 1, 12), (2, 2, 7)])
@pytest.mark.parametrize("kappa_kind", ["p1", "none", "const"])
def test_diffusion_matrix_fp64(orc, tdim, deg, n, kappa_kind):
    case = Case(orc, tdim, n, jitter=0.15, seed=1)
    V = d2.FunctionSpace(case.mesh, "Lagrange", deg)
    W = d2.FunctionSpace(case.mesh, "Lagrange", 1)
    u, v = d2.TrialFunction(V), d2.TestFunction(V)
    kv = synthetic.uniform_field(case.om.nv, 0.5, 2.0, seed=2)
    if kappa_kind == "p1":
        kappa = d2.Function(W, kv)
        a = kappa * d2.inner(d2.grad(u), d2.grad(v)) * d2.dx
        okw = dict(w=kv, coeff=2)
    elif kappa_kind == "none":
        a = d2.inner(d2.grad(u), d2.grad(v)) * d2.dx
        okw = dict()
    else:
        a = d2.Constant(1.7) * d2.inner(d2.grad(u), d2.grad(v)) * d2.dx
        okw = dict(coeff=1, c=(1.7,))
    A = d2.assemble(a)
    rp, cols, vals = A.data()
    ref, od, N = _oracle_matrix(orc, case, orc.DIFFUSION, deg, 1, rp, cols, **okw)
    orp, ocols = orc.sparsity(N, N, od, od)
    assert np.array_equal(rp, orp) and np.array_equal(cols, ocols)
    assert row_scaled_err(rp, vals, ref) <= FP64_TOL


@pytest.mark.parametrize("tdim,deg,n", [(3, 1, 5), (3, 2, 3), (2, 2, 6)])
def test_diffusion_fp32_contraction(orc, tdim, deg, n):
    case = Case(orc, tdim, n, jitter=0.15, seed=3)
    V = d2.FunctionSpace(case.mesh, "Lagrange", deg)
    W = d2.FunctionSpace(case.mesh, "Lagrange", 1)
    kv = synthetic.uniform_field(case.om.nv, 0.5, 2.0, seed=4)
    kappa = d2.Function(W, kv)
    u, v = d2.TrialFunction(V), d2.TestFunction(V)
    A = d2.assemble(kappa * d2.inner(d2.grad(u), d2.grad(v)) * d2.dx, precision="fp32")
    rp, cols, vals = A.data()
    ref, _, _ = _oracle_matrix(orc, case, orc.DIFFUSION, deg, 1, rp, cols, w=kv, coeff=2)
    err = row_scaled_err(rp, vals, ref)
    assert err <= FP32_TOL and err > 0.0  # genuinely computed in fp32


@pytest.mark.parametrize("deg,n", [(1, 3), (2, 2)])
@pytest.mark.parametrize("precision,tol", [("fp64", FP64_TOL), ("fp32", FP32_TOL)])
def test_elasticity_system(orc, deg, n, precision, tol):
    case = Case(orc, 3, n, jitter=0.15, seed=5)
    V = d2.VectorFunctionSpace(case.mesh, "Lagrange", deg)
    u, v = d2.TrialFunction(V), d2.TestFunction(V)
    E, nu = 1.0, 0.3
    mu = d2.Constant(E / (2 * (1 + nu)))
    lmbda = d2.Constant(E * nu / ((1 + nu) * (1 - 2 * nu)))
    eps = lambda w: d2.sym(d2.grad(w))
    sigma = lambda w: 2 * mu * eps(w) + lmbda * d2.tr(eps(w)) * d2.Identity(3)
    a = d2.inner(sigma(u), eps(v)) * d2.dx
    L = d2.inner(d2.Constant((0.0, 0.0, -1.0)), v) * d2.dx
    A, b = d2.assemble_system(a, L, precision=precision)
    rp, cols, vals = A.data()
    ref, od, N = _oracle_matrix(orc, case, orc.ELASTICITY, deg, 3, rp, cols, mu=float(mu),
                                lm=float(lmbda))
    orp, ocols = orc.sparsity(N, N, od, od)
    assert np.array_equal(rp, orp) and np.array_equal(cols, ocols)
    assert row_scaled_err(rp, vals, ref) <= tol
    fL = orc.form(orc.LOAD, 3, deg, 3, coeff=1, c=(0.0, 0.0, -1.0))
    bref = orc.assemble_vector(fL, case.om, od, N)
    assert vec_err(b.get_local(), bref) <= FP64_TOL


@pytest.mark.parametrize("tdim,deg,n", [(3, 1, 5), (3, 2, 3), (2, 1, 9), (2, 2, 6)])
def test_system_and_vector_p1_load(orc, tdim, deg, n):
    case = Case(orc, tdim, n, jitter=0.1, seed=6)
    V = d2.FunctionSpace(case.mesh, "Lagrange", deg)
    W = d2.FunctionSpace(case.mesh, "Lagrange", 1)
    kv = synthetic.uniform_field(case.om.nv, 0.5, 2.0, seed=7)
    fv = synthetic.uniform_field(case.om.nv, -1.0, 1.0, seed=8)
    kappa, f = d2.Function(W, kv), d2.Function(W, fv)
    u, v = d2.TrialFunction(V), d2.TestFunction(V)
    a = kappa * d2.inner(d2.grad(u), d2.grad(v)) * d2.dx
    L = f * v * d2.dx
    A, b = d2.assemble_system(a, L)
    b2 = d2.assemble(L)
    rp, cols, vals = A.data()
    ref, od, N = _oracle_matrix(orc, case, orc.DIFFUSION, deg, 1, rp, cols, w=kv, coeff=2)
    assert row_scaled_err(rp, vals, ref) <= FP64_TOL
    bref = orc.assemble_vector(orc.form(orc.LOAD, tdim, deg, 1, coeff=2), case.om, od, N, w=fv)
    assert vec_err(b.get_local(), bref) <= FP64_TOL
    assert vec_err(b2.get_local(), bref) <= FP64_TOL


def test_reference_tetrahedron_known_answer():
    # python/test/unit/fem/test_assembler.py:351-387 on the engine itself.
    m = d2.Mesh(np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]], float),
                np.array([[0, 1, 2, 3]], np.uint32))
    V = d2.FunctionSpace(m, "Lagrange", 1)
    u, v = d2.TrialFunction(V), d2.TestFunction(V)
    A = d2.assemble(d2.dot(d2.grad(v), d2.grad(u)) * d2.dx).array()
    A0 = np.array([[1 / 2, -1 / 6, -1 / 6, -1 / 6], [-1 / 6, 1 / 6, 0, 0],
                   [-1 / 6, 0, 1 / 6, 0], [-1 / 6, 0, 0, 1 / 6]])
    assert round(np.linalg.norm(A - A0), 7) == 0


def test_add_values_and_reuse(orc):
    case = Case(orc, 3, 3)
    V = d2.FunctionSpace(case.mesh, "Lagrange", 2)
    u, v = d2.TrialFunction(V), d2.TestFunction(V)
    a = d2.inner(d2.grad(u), d2.grad(v)) * d2.dx
    A = d2.assemble(a)
    first = A.data()[2].copy()
    d2.assemble(a, tensor=A, add_values=True)
    assert np.allclose(A.data()[2], 2 * first, rtol=1e-15, atol=0)
    d2.assemble(a, tensor=A)  # reassembly zeroes first (AssemblerBase.cpp:194-195)
    assert np.array_equal(A.data()[2], first)


def test_deterministic_bitwise(orc):
    case = Case(orc, 3, 4, jitter=0.15, seed=9)
    V = d2.VectorFunctionSpace(case.mesh, "Lagrange", 2)
    u, v = d2.TrialFunction(V), d2.TestFunction(V)
    a = d2.inner(d2.sym(d2.grad(u)), d2.sym(d2.grad(v))) * d2.dx
    A1 = d2.assemble(a).data()[2]
    V.pattern().retile(64, 16 * 1024)  # different launch shape, same result bits
    A2 = d2.assemble(a).data()[2]
    assert np.array_equal(A1, A2)


def test_assembly_on_a_user_stream_is_joined():
    """The tile classes run on side streams forked from the caller's stream and
    joined back to it: work queued on that stream right after the call sees
    the finished matrix, and the values equal the default-stream assembly."""
    mesh = d2.UnitCubeMesh(24, 24, 24)
    V = d2.FunctionSpace(mesh, "Lagrange", 2)
    W = d2.FunctionSpace(mesh, "Lagrange", 1)
    kappa = d2.Function(W, synthetic.uniform_field(mesh.num_vertices(), 0.5, 2.0, seed=3))
    f = d2.Function(W, synthetic.uniform_field(mesh.num_vertices(), -1.0, 1.0, seed=4))
    u, v = d2.TrialFunction(V), d2.TestFunction(V)
    a = kappa * d2.inner(d2.grad(u), d2.grad(v)) * d2.dx
    L = f * v * d2.dx
    A0, b0 = d2.assemble_system(a, L)
    ref_vals, ref_b = A0.values_tensor().clone(), b0.tensor().clone()
    torch.cuda.synchronize()
    s = torch.cuda.Stream()
    S = d2.SystemAssembler(a, L)
    with torch.cuda.stream(s):
        A1, b1 = S.assemble()
        snap_vals = A1.values_tensor().clone()  # queued on s, no host sync before it
        snap_b = b1.tensor().clone()
    torch.cuda.synchronize()
    assert torch.equal(snap_vals, ref_vals) and torch.equal(snap_b, ref_b)


@pytest.mark.parametrize("tdim,deg,vs,n", [(3, 1, 1, 5), (3, 2, 1, 3), (3, 2, 3, 3), (2, 2, 1, 7),
                                            (2, 1, 1, 9), (3, 1, 3, 4), (3, 2, 0, 3), (2, 2, 0, 6)])
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_matrix_free_action_matches_csr(orc, tdim, deg, vs, n, precision):
    """vs = 0: scalar space with a constant coefficient."""
    case = Case(orc, tdim, n, jitter=0.1, seed=10)
    V = d2.FunctionSpace(case.mesh, "Lagrange", deg, value_size=max(vs, 1))
    u, v = d2.TrialFunction(V), d2.TestFunction(V)
    if vs == 0:
        a = d2.Constant(1.7) * d2.inner(d2.grad(u), d2.grad(v)) * d2.dx
    elif vs == 1:
        W = d2.FunctionSpace(case.mesh, "Lagrange", 1)
        kappa = d2.Function(W, synthetic.uniform_field(case.om.nv, 0.5, 2.0, seed=11))
        a = kappa * d2.inner(d2.grad(u), d2.grad(v)) * d2.dx
    else:
        a = d2.inner(2.0 * d2.sym(d2.grad(u)) + 0.5 * d2.tr(d2.grad(u)) * d2.Identity(3),
                     d2.sym(d2.grad(v))) * d2.dx
    x = torch.randn(V.dim(), dtype=torch.float64, device="cuda", generator=torch.Generator("cuda").manual_seed(0))
    y = d2.assemble_action(a, d2.Vector(x), precision=precision).get_local()
    A = d2.assemble(a).sparray()
    yref = A @ x.cpu().numpy()
    tol = FP64_TOL * 10 if precision == "fp64" else FP32_TOL * 10
    assert vec_err(y, yref) <= tol
    # the per-row sums run in a fixed order: a second action is bitwise equal
    y2 = d2.assemble_action(a, d2.Vector(x), precision=precision).get_local()
    assert np.array_equal(y, y2)


@pytest.mark.parametrize("tdim,deg", [(3, 1), (3, 2), (2, 2)])
def test_vjp_matches_central_differences(orc, tdim, deg):
    """dL/dkappa of L(kappa) = <gA, A(kappa)> for A = kappa*grad(u).grad(v)*dx
    against central differences (h = 1e-6) of the engine's own forward
    assembly on 64 random directions; error scaled by |dL/dkappa| |dir|."""
    from dolfin_b200.autodiff import vjp_kappa
    case = Case(orc, tdim, 4 if tdim == 3 else 8, jitter=0.1, seed=21)
    V = d2.FunctionSpace(case.mesh, "Lagrange", deg)
    W = d2.FunctionSpace(case.mesh, "Lagrange", 1)
    u, v = d2.TrialFunction(V), d2.TestFunction(V)
    nv = case.om.nv
    kv = synthetic.lognormal_field(nv, 0.5, seed=22)
    P = V.pattern()
    gA = torch.randn(P.nnz(), dtype=torch.float64, device="cuda",
                     generator=torch.Generator("cuda").manual_seed(23))
    kt = torch.as_tensor(kv, device="cuda")
    dk = vjp_kappa(V, kt, gA)

    def L(kvals):
        kappa = d2.Function(W, kvals)
        A = d2.assemble(kappa * d2.inner(d2.grad(u), d2.grad(v)) * d2.dx)
        return float(torch.dot(gA, A.values_tensor()))

    h = 1e-6
    dirs = torch.randn(64, nv, dtype=torch.float64, device="cuda",
                       generator=torch.Generator("cuda").manual_seed(24))
    worst = 0.0
    for d in dirs:
        fd = (L(kt + h * d) - L(kt - h * d)) / (2 * h)
        ad = float(torch.dot(dk, d))
        worst = max(worst, abs(fd - ad) / (float(dk.norm()) * float(d.norm())))
    assert worst <= 1e-8


@pytest.mark.parametrize("deg", [1, 2])
def test_vjp_matches_oracle_derivative_form(orc, deg):
    from dolfin_b200.autodiff import vjp_kappa
    case = Case(orc, 3, 3, jitter=0.1, seed=12)
    V = d2.FunctionSpace(case.mesh, "Lagrange", deg)
    W = d2.FunctionSpace(case.mesh, "Lagrange", 1)
    rng = np.random.default_rng(13)
    kv = synthetic.lognormal_field(case.om.nv, 0.5, seed=14)
    fv = synthetic.uniform_field(case.om.nv, -1.0, 1.0, seed=15)
    P = V.pattern()
    gA = rng.standard_normal(P.nnz())
    gb = rng.standard_normal(V.dim())
    dk = vjp_kappa(V, torch.as_tensor(kv, device="cuda"), torch.as_tensor(gA, device="cuda"),
                   f=torch.as_tensor(fv, device="cuda"), gb=torch.as_tensor(gb, device="cuda"))
    rp, cols = P.csr_host()
    od, _ = orc.dofmap(case.om, deg, 1)
    ref = orc.vjp_diffusion(orc.form(orc.DIFFUSION, 3, deg, 1, coeff=2), case.om, od, rp, cols, gA,
                            f=fv, gb=gb, load_has_kappa=True)
    assert vec_err(dk.cpu().numpy(), ref) <= 1e-12
