"""Entry-wise parity with the oracle at the benchmark configurations' full
sizes.

Each test assembles one benchmark configuration on the GPU and compares it
entry by entry with the oracle (the CPU restatement of DOLFIN's serial
assembly) on the same mesh and coefficients: dofmap, CSR row pointers and
columns bit-exact; FP64 values within 1e-12 row-scaled
(|A_ij - R_ij| <= 1e-12 max_j |R_ij|), vectors within 1e-12 of max |b|;
the FP32-contraction path within 1e-6 on the same scale.  The large
configurations run the oracle by row blocks on all host cores
(oracle/parallel.py), which gives exactly its whole-mesh rows.

  * P1 Poisson A+b, UnitCubeMesh(32) (196,608 cells)
  * vector P2 elasticity A+b, UnitCubeMesh(48) jittered (231,797,385 nnz),
    plus the matrix-free action against the oracle's CSR
  * P2 Poisson A+b, UnitCubeMesh(96) (204,763,393 nnz), plus the action
  * the adjoint dL/dkappa on P1 UnitCubeMesh(32): against the oracle's
    derivative-form assembly and against central differences
  * 32 members of the batched workload's own spec (UnitSquareMesh(n),
    n log-uniform in [8, 256]) in one persistent launch
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = [pytest.mark.gpu,
              pytest.mark.filterwarnings("ignore:Sparse CSR tensor support is in beta")]

import dolfin_b200 as d2
from dolfin_b200 import synthetic

FP64_TOL = 1e-12
FP32_TOL = 1e-6


def row_scaled_err(rp, vals, ref):
    """max |vals - ref| / (max |ref| of the row), over all entries."""
    rowmax = np.maximum.reduceat(np.abs(ref), rp[:-1].astype(np.int64))
    rowmax[rowmax == 0] = 1.0
    lens = np.diff(rp)
    worst = 0.0
    # chunked over rows to bound the temporaries at full size
    step = 1 << 20
    for r0 in range(0, len(lens), step):
        r1 = min(len(lens), r0 + step)
        a, b = int(rp[r0]), int(rp[r1])
        s = np.repeat(rowmax[r0:r1], lens[r0:r1])
        worst = max(worst, float(np.max(np.abs(vals[a:b] - ref[a:b]) / s)))
    return worst


def vec_err(b, ref):
    return float(np.max(np.abs(b - ref)) / max(float(np.max(np.abs(ref))), 1e-300))


def _poisson(n, deg, seed, jitter=0.0):
    mesh = d2.UnitCubeMesh(n, n, n)
    from oracle import oracle as orc
    om = orc.unit_cube_mesh(n, n, n)
    if jitter:
        x = synthetic.jitter_interior(om.coords, n, jitter, seed)
        mesh.set_coordinates(x)
        om.coords = x
    V = d2.FunctionSpace(mesh, "Lagrange", deg)
    W = d2.FunctionSpace(mesh, "Lagrange", 1)
    kv = synthetic.uniform_field(om.nv, 0.5, 2.0, seed + 1)
    fv = synthetic.uniform_field(om.nv, -1.0, 1.0, seed + 2)
    kappa, f = d2.Function(W, kv), d2.Function(W, fv)
    u, v = d2.TrialFunction(V), d2.TestFunction(V)
    a = kappa * d2.inner(d2.grad(u), d2.grad(v)) * d2.dx
    L = f * v * d2.dx
    return mesh, om, V, a, L, kv, fv


def _check_dofmap(orc, om, V, deg, bs):
    od, N = orc.dofmap(om, deg, bs)
    assert N == V.dim()
    assert np.array_equal(V.dofmap().cell_dofs_all(), od)
    return od, N


def _action_err(A_rp, A_cols, ref_vals, x, y):
    """|y - R x| per row, scaled by sum_j |R_ij x_j| of the row (the size of
    the terms the action sums)."""
    import scipy.sparse as sp
    n = len(A_rp) - 1
    R = sp.csr_matrix((ref_vals, A_cols, A_rp), shape=(n, n))
    yref = R @ x
    mag = abs(R) @ np.abs(x)
    mag[mag == 0] = 1.0
    return float(np.max(np.abs(y - yref) / mag))


def test_config1_p1_poisson_full(orc):
    n = 32
    mesh, om, V, a, L, kv, fv = _poisson(n, 1, 100)
    od, N = _check_dofmap(orc, om, V, 1, 1)
    A, b = d2.assemble_system(a, L)
    rp, cols, vals = A.data()
    orp, ocols = orc.sparsity(N, N, od, od)
    assert np.array_equal(rp, orp) and np.array_equal(cols, ocols)
    assert len(cols) == 15 * n**3 + 21 * n**2 + 9 * n + 1
    ref = orc.assemble_matrix(orc.form(orc.DIFFUSION, 3, 1, 1, coeff=orc.COEFF_P1), om, od, od,
                              orp, ocols, w=kv)
    bref = orc.assemble_vector(orc.form(orc.LOAD, 3, 1, 1, coeff=orc.COEFF_P1), om, od, N, w=fv)
    assert row_scaled_err(rp, vals, ref) <= FP64_TOL
    assert vec_err(b.get_local(), bref) <= FP64_TOL
    A32, b32 = d2.assemble_system(a, L, precision="fp32")
    assert row_scaled_err(rp, A32.values_tensor().cpu().numpy(), ref) <= FP32_TOL
    assert vec_err(b32.get_local(), bref) <= FP64_TOL  # the load stays FP64


def _parallel_reference(orc, om, od, N, bs, deg, rp, a, L, wa=None, wL=None):
    from oracle import parallel
    ocols, ovals, ob, bad, _ = parallel.assemble_rows(
        om, od, N, bs, 4 if deg == 1 else 10, rp, a=a, L=L, wa=wa, wL=wL,
        nvert=om.nv if deg == 2 else None)
    assert bad == 0, f"{bad} rows differ in length from the oracle's"
    return ocols, ovals, ob


def test_config2_elasticity_full(orc):
    n = 48
    mesh = d2.UnitCubeMesh(n, n, n)
    om = orc.unit_cube_mesh(n, n, n)
    x = synthetic.jitter_interior(om.coords, n, 0.15, 200)
    mesh.set_coordinates(x)
    om.coords = x
    V = d2.VectorFunctionSpace(mesh, "Lagrange", 2)
    u, v = d2.TrialFunction(V), d2.TestFunction(V)
    E, nu = 1.0, 0.3
    mu, lm = E / (2 * (1 + nu)), E * nu / ((1 + nu) * (1 - 2 * nu))
    eps = lambda w: d2.sym(d2.grad(w))
    a = d2.inner(2 * d2.Constant(mu) * eps(u) + d2.Constant(lm) * d2.tr(eps(u)) * d2.Identity(3),
                 eps(v)) * d2.dx
    L = d2.inner(d2.Constant((0.0, 0.0, -1.0)), v) * d2.dx
    od, N = _check_dofmap(orc, om, V, 2, 3)
    A, b = d2.assemble_system(a, L)
    rp, cols, vals = A.data()
    assert len(cols) == 9 * (230 * n**3 + 138 * n**2 + 24 * n + 1)
    fa = dict(kind=orc.ELASTICITY, tdim=3, degree0=2, vsize0=3, mu=mu, lmbda=lm)
    fl = dict(kind=orc.LOAD, tdim=3, degree0=2, vsize0=3, coeff=orc.COEFF_CONST, c=(0.0, 0.0, -1.0))
    ocols, ovals, ob = _parallel_reference(orc, om, od, N, 3, 2, rp, fa, fl)
    assert np.array_equal(cols, ocols)
    assert row_scaled_err(rp, vals, ovals) <= FP64_TOL
    assert vec_err(b.get_local(), ob) <= FP64_TOL
    del vals
    A32, _ = d2.assemble_system(a, L, precision="fp32")
    assert row_scaled_err(rp, A32.values_tensor().cpu().numpy(), ovals) <= FP32_TOL
    del A32
    # matrix-free action y = A x against the oracle's CSR
    xv = np.random.default_rng(201).standard_normal(N)
    y = d2.assemble_action(a, d2.Vector(torch.as_tensor(xv, device="cuda"))).get_local()
    assert _action_err(rp, cols, ovals, xv, y) <= 1e-12


def test_config5_p2_poisson_full(orc):
    n = 96
    mesh, om, V, a, L, kv, fv = _poisson(n, 2, 500)
    od, N = _check_dofmap(orc, om, V, 2, 1)
    assert N == (2 * n + 1) ** 3
    A, b = d2.assemble_system(a, L)
    rp, cols, vals = A.data()
    assert len(cols) == 230 * n**3 + 138 * n**2 + 24 * n + 1
    fa = dict(kind=orc.DIFFUSION, tdim=3, degree0=2, coeff=orc.COEFF_P1)
    fl = dict(kind=orc.LOAD, tdim=3, degree0=2, coeff=orc.COEFF_P1)
    ocols, ovals, ob = _parallel_reference(orc, om, od, N, 1, 2, rp, fa, fl, wa=kv, wL=fv)
    assert np.array_equal(cols, ocols)
    assert row_scaled_err(rp, vals, ovals) <= FP64_TOL
    assert vec_err(b.get_local(), ob) <= FP64_TOL
    del vals
    A32, _ = d2.assemble_system(a, L, precision="fp32")
    assert row_scaled_err(rp, A32.values_tensor().cpu().numpy(), ovals) <= FP32_TOL
    del A32
    xv = np.random.default_rng(501).standard_normal(N)
    y = d2.assemble_action(a, d2.Vector(torch.as_tensor(xv, device="cuda"))).get_local()
    assert _action_err(rp, cols, ovals, xv, y) <= 1e-12
    y32 = d2.assemble_action(a, d2.Vector(torch.as_tensor(xv, device="cuda")), precision="fp32").get_local()
    assert _action_err(rp, cols, ovals, xv, y32) <= FP32_TOL
    ytc = d2.assemble_action(a, d2.Vector(torch.as_tensor(xv, device="cuda")), precision="fp32_tc").get_local()
    assert _action_err(rp, cols, ovals, xv, ytc) <= FP32_TOL


@pytest.mark.parametrize("precision,tol_oracle,tol_fd", [("fp64", 1e-12, 1e-8), ("fp32", 1e-6, 1e-6)])
def test_config4_adjoint_n32(orc, precision, tol_oracle, tol_fd):
    """dL/dkappa of L(kappa) = <gA, A(kappa)> + <gb, b(kappa)>, A =
    kappa*grad(u).grad(v)*dx, b = kappa*f*v*dx, kappa = exp(g), g ~ N(0,
    0.5^2), gA, gb ~ N(0, 1): against the oracle's FP64 derivative-form
    assembly, and (A part) against central differences (h = 1e-6) of the
    engine's FP64 forward assembly on 64 random directions, error scaled by
    |dL/dkappa| |direction|.  The FP32-contraction adjoint is held to 1e-6
    against both."""
    from dolfin_b200.autodiff import vjp_kappa
    n = 32
    mesh = d2.UnitCubeMesh(n, n, n)
    om = orc.unit_cube_mesh(n, n, n)
    V = d2.FunctionSpace(mesh, "Lagrange", 1)
    u, v = d2.TrialFunction(V), d2.TestFunction(V)
    nv = om.nv
    kv = synthetic.lognormal_field(nv, 0.5, 400)
    fv = synthetic.uniform_field(nv, -1.0, 1.0, 401)
    P = V.pattern()
    g = torch.Generator("cuda").manual_seed(402)
    gA = torch.randn(P.nnz(), dtype=torch.float64, device="cuda", generator=g)
    gb = torch.randn(V.dim(), dtype=torch.float64, device="cuda", generator=g)
    kt = torch.as_tensor(kv, device="cuda")
    ft = torch.as_tensor(fv, device="cuda")
    dk = vjp_kappa(V, kt, gA, f=ft, gb=gb, precision=precision)
    rp, cols = P.csr_host()
    od, _ = orc.dofmap(om, 1, 1)
    ref = orc.vjp_diffusion(orc.form(orc.DIFFUSION, 3, 1, 1, coeff=orc.COEFF_P1), om, od, rp, cols,
                            gA.cpu().numpy(), f=fv, gb=gb.cpu().numpy(), load_has_kappa=True)
    assert vec_err(dk.cpu().numpy(), ref) <= tol_oracle
    dkA = vjp_kappa(V, kt, gA, precision=precision)  # the A part alone
    W = V
    A = d2.Matrix()

    def L_of(kvals):
        kappa = d2.Function(W, kvals)
        d2.assemble(kappa * d2.inner(d2.grad(u), d2.grad(v)) * d2.dx, tensor=A)
        return float(torch.dot(gA, A.values_tensor()))

    h = 1e-6
    dirs = torch.randn(64, nv, dtype=torch.float64, device="cuda", generator=g)
    worst = 0.0
    for d in dirs:
        fd = (L_of(kt + h * d) - L_of(kt - h * d)) / (2 * h)
        ad = float(torch.dot(dkA, d))
        worst = max(worst, abs(fd - ad) / (float(dkA.norm()) * float(d.norm())))
    assert worst <= tol_fd


def test_config3_batched_real_sizes(orc):
    """32 members (every 16th) of the 512-mesh batched workload's own seeded
    spec: n log-uniform in [8, 256], degree 1 or 2, jitter 0.2h."""
    from dolfin_b200.batch import BatchAssembler
    specs = synthetic.batched_square_meshes(512, 2024)[::16]
    assert len(specs) == 32 and max(s["n"] for s in specs) > 100
    built = [synthetic.build_batch_member(s) for s in specs]
    B = BatchAssembler([(V, k) for (_, V, k, _, _) in built])
    mats = [A.values_tensor().cpu().numpy() for A in B.assemble()]
    m32 = [A.values_tensor().cpu().numpy() for A in B.assemble("fp32")]
    for spec, (mesh, V, k, x, kv), vals, v32 in zip(specs, built, mats, m32):
        om = orc.unit_square_mesh(spec["n"], spec["n"])
        om.coords = x
        od, N = orc.dofmap(om, spec["degree"])
        assert np.array_equal(V.dofmap().cell_dofs_all(), od)
        rp, cols = V.pattern().csr_host()
        orp, ocols = orc.sparsity(N, N, od, od)
        assert np.array_equal(rp, orp) and np.array_equal(cols, ocols)
        ref = orc.assemble_matrix(orc.form(orc.DIFFUSION, 2, spec["degree"], 1, coeff=orc.COEFF_P1),
                                  om, od, od, rp, cols, w=kv)
        assert row_scaled_err(rp, vals, ref) <= FP64_TOL
        assert row_scaled_err(rp, v32, ref) <= FP32_TOL
