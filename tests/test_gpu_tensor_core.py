"""The tensor-core (tcgen05) FP32-contraction matrix-free action (precision
"fp32_tc") of
kappa*grad(u).grad(v)*dx on P2 tetrahedra against the oracle's CSR times x:
|y - R x| <= 1e-6 sum_j |R_ij x_j| per row, with a P1 kappa and with a
constant one, on meshes whose cell count is and is not a multiple of the
128-cell tile; bitwise repeatable; no tensor-core wait ran out."""
import ctypes as C

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import dolfin_b200 as d2
from dolfin_b200 import _capi, synthetic


def _status():
    s = C.c_int(-1)
    _capi.call("db2_tensor_core_status", C.byref(s))
    return s.value


@pytest.mark.parametrize("n", [4, 5])
@pytest.mark.parametrize("kappa_kind", ["p1", "const"])
def test_tensor_core_action_matches_oracle(orc, n, kappa_kind):
    import scipy.sparse as sp
    mesh = d2.UnitCubeMesh(n, n, n)
    om = orc.unit_cube_mesh(n, n, n)
    x = synthetic.jitter_interior(om.coords, n, 0.15, 40)
    mesh.set_coordinates(x)
    om.coords = x
    V = d2.FunctionSpace(mesh, "Lagrange", 2)
    W = d2.FunctionSpace(mesh, "Lagrange", 1)
    u, v = d2.TrialFunction(V), d2.TestFunction(V)
    kv = synthetic.lognormal_field(om.nv, 0.5, 41)
    if kappa_kind == "p1":
        a = d2.Function(W, kv) * d2.inner(d2.grad(u), d2.grad(v)) * d2.dx
        okw = dict(w=kv, coeff=orc.COEFF_P1)
    else:
        a = d2.Constant(2.5) * d2.inner(d2.grad(u), d2.grad(v)) * d2.dx
        okw = dict(coeff=orc.COEFF_CONST, c=(2.5,))
    od, N = orc.dofmap(om, 2, 1)
    rp, cols = V.pattern().csr_host()
    ref = orc.assemble_matrix(orc.form(orc.DIFFUSION, 3, 2, 1, coeff=okw["coeff"], c=okw.get("c", (0, 0, 0))),
                              om, od, od, rp, cols, w=okw.get("w"))
    R = sp.csr_matrix((ref, cols, rp), shape=(N, N))
    xv = np.random.default_rng(42).standard_normal(N)
    xt = d2.Vector(torch.as_tensor(xv, device="cuda"))
    y = d2.assemble_action(a, xt, precision="fp32_tc").get_local()
    y2 = d2.assemble_action(a, xt, precision="fp32_tc").get_local()
    assert _status() == 0
    assert np.array_equal(y, y2)
    mag = abs(R) @ np.abs(xv)
    err = float(np.max(np.abs(y - R @ xv) / mag))
    assert err <= 1e-6, err
    # and it is the tensor-core path, neither the FP64 one nor the FP32
    # quadrature one: they differ
    y64 = d2.assemble_action(a, xt).get_local()
    assert float(np.max(np.abs(y64 - R @ xv) / mag)) <= 1e-12
    assert not np.array_equal(y, y64)
    y32 = d2.assemble_action(a, xt, precision="fp32").get_local()
    assert float(np.max(np.abs(y32 - R @ xv) / mag)) <= 1e-6
    assert not np.array_equal(y, y32) and not np.array_equal(y32, y64)
