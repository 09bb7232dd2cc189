"""The allocation-free adjoint entry point (db2_vjp_kappa_noalloc).

It exists for callers that cannot let the engine allocate device memory
during a call -- applications that own all device memory through their own
pool allocator, or loops whose concurrently running streams cudaMalloc's
implicit synchronisation would stall.  This file is named to be collected
last: it checks the entry point, called through the C ABI, against the
allocating entry point (db2_vjp_kappa) on two calls in a row, and that those
two calls leave the device's free memory unchanged, both when run alone in a
fresh process and after the rest of the suite."""
import ctypes as C

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import dolfin_b200 as d2
from dolfin_b200 import _capi, synthetic


def _vjp(name, P, kappa, f, gA, gb, dk):
    a = _capi.make_form(_capi.FORM_DIFFUSION, _capi.COEFF_P1_SCALED, (1.0,))
    L = _capi.make_form(_capi.FORM_LOAD, _capi.COEFF_P1_SCALED, (1.0,))
    p = lambda t: C.c_void_p(t.data_ptr())
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    _capi.call(name, P.handle, C.byref(a), p(kappa), C.byref(L), p(f), p(gA), p(gb),
               _capi.FP64, p(dk), stream)


@pytest.mark.parametrize("deg", [1, 2])
def test_noalloc_vjp_matches_allocating_entry_point_twice(deg):
    n = 6
    mesh = d2.UnitCubeMesh(n, n, n)
    mesh.set_coordinates(synthetic.jitter_interior(mesh.coordinates(), n, 0.1, 5))
    V = d2.FunctionSpace(mesh, "Lagrange", deg)
    P = V.pattern()
    rng = np.random.default_rng(6)
    nv = mesh.num_vertices()
    kappa = torch.as_tensor(synthetic.lognormal_field(nv, 0.5, 7), device="cuda")
    f = torch.as_tensor(rng.uniform(-1, 1, nv), device="cuda")
    # an ordinary assembly makes the pattern resident on the device (which
    # also sets up the entry point's fixed array there)
    u, v = d2.TrialFunction(V), d2.TestFunction(V)
    d2.assemble(d2.inner(d2.grad(u), d2.grad(v)) * d2.dx)
    gA = torch.as_tensor(rng.standard_normal(P.nnz()), device="cuda")
    gb = torch.as_tensor(rng.standard_normal(V.dim()), device="cuda")
    outs = [torch.full((nv,), float("nan"), dtype=torch.float64, device="cuda") for _ in range(2)]
    ref = torch.empty(nv, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for out in outs:
        _vjp("db2_vjp_kappa_noalloc", P, kappa, f, gA, gb, out)
        torch.cuda.synchronize()
    # nothing was allocated on the device by the two calls
    assert torch.cuda.mem_get_info()[0] == free0
    _vjp("db2_vjp_kappa", P, kappa, f, gA, gb, ref)
    torch.cuda.synchronize()
    for out in outs:
        err = float((out - ref).abs().max() / ref.abs().max())
        assert err <= 1e-12


def test_noalloc_vjp_rejects_patterns_beyond_its_array():
    mesh = d2.UnitCubeMesh(45, 45, 45)  # 546,750 tetrahedra > 524,288
    V = d2.FunctionSpace(mesh, "Lagrange", 1)
    P = V.pattern()
    nv = mesh.num_vertices()
    z = torch.zeros(max(nv, P.nnz()), dtype=torch.float64, device="cuda")
    with pytest.raises(_capi.DB2Error) as exc:
        _vjp("db2_vjp_kappa_noalloc", P, z, z, z, z, z)
    assert exc.value.code == 2 and "2097152" in str(exc.value)
