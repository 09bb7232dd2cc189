"""The C++ drop-in classes (GpuAssembler, GpuSystemAssembler of
include/dolfin_b200_assembler.h, built as libdolfin_b200_cpp.so) driven from
a compiled C++ program (tests/cpp/shim_driver.cpp, built by the engine's
Makefile) agree with the Python path on the same inputs: CSR structure and
values bitwise for the scalar system assemblies (with and without ds terms
and a Dirichlet condition) and add_values, elasticity within 1e-14
row-scaled (its Lame constants reach the Python path through the form
recogniser's fit), and a wrong-size tensor is refused with DOLFIN's
message."""
import os
import subprocess

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import dolfin_b200 as d2
from dolfin_b200 import synthetic

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DRIVER = os.path.join(ROOT, "dolfin_b200", "_lib", "shim_driver")


def _read(d, name, dtype):
    return np.fromfile(os.path.join(d, name), dtype=dtype)


def _matrix(d, case):
    return (_read(d, f"{case}_rowptr.bin", np.int32), _read(d, f"{case}_cols.bin", np.int32),
            _read(d, f"{case}_vals.bin", np.float64))


def test_cpp_shim_matches_python_path(tmp_path):
    assert os.path.exists(DRIVER), "build the engine first (make -C dolfin_b200/csrc)"
    n = 4
    mesh = d2.UnitCubeMesh(n, n, n)
    x = synthetic.jitter_interior(mesh.coordinates(), n, 0.15, 61)
    mesh.set_coordinates(x)
    nv = mesh.num_vertices()
    kv = synthetic.uniform_field(nv, 0.5, 2.0, 62)
    fv = synthetic.uniform_field(nv, -1.0, 1.0, 63)
    ind, outd = tmp_path / "in", tmp_path / "out"
    ind.mkdir()
    outd.mkdir()
    x.astype(np.float64).tofile(ind / "coords.bin")
    kv.tofile(ind / "kappa.bin")
    fv.tofile(ind / "f.bin")
    r = subprocess.run([DRIVER, str(n), str(ind), str(outd)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr

    P1 = d2.FunctionSpace(mesh, "Lagrange", 1)
    P2 = d2.FunctionSpace(mesh, "Lagrange", 2)
    kappa, f = d2.Function(P1, kv), d2.Function(P1, fv)
    u, v = d2.TrialFunction(P2), d2.TestFunction(P2)

    A, b = d2.SystemAssembler(kappa * d2.inner(d2.grad(u), d2.grad(v)) * d2.dx, f * v * d2.dx).assemble()
    for got, ref in zip(_matrix(outd, "system"), A.data()):
        assert np.array_equal(got, ref)
    assert np.array_equal(_read(outd, "system_b.bin", np.float64), b.get_local())

    a = kappa * d2.inner(d2.grad(u), d2.grad(v)) * d2.dx + d2.Constant(0.5) * u * v * d2.ds
    L = f * v * d2.dx + d2.Constant(1.5) * v * d2.ds
    bc = d2.DirichletBC(P2, 0.25, lambda p, on: on and p[0] < 1e-12)
    A, b = d2.SystemAssembler(a, L, bc).assemble()
    for got, ref in zip(_matrix(outd, "system_bc"), A.data()):
        assert np.array_equal(got, ref)
    assert np.array_equal(_read(outd, "system_bc_b.bin", np.float64), b.get_local())

    V = d2.VectorFunctionSpace(mesh, "Lagrange", 2)
    u3, v3 = d2.TrialFunction(V), d2.TestFunction(V)
    E, nu = 1.0, 0.3
    mu, lm = d2.Constant(E / (2 * (1 + nu))), d2.Constant(E * nu / ((1 + nu) * (1 - 2 * nu)))
    eps = lambda w: d2.sym(d2.grad(w))
    A = d2.assemble(d2.inner(2 * mu * eps(u3) + lm * d2.tr(eps(u3)) * d2.Identity(3), eps(v3)) * d2.dx)
    b = d2.assemble(d2.inner(d2.Constant((0.0, 0.0, -1.0)), v3) * d2.dx)
    rp, cols, vals = _matrix(outd, "elasticity")
    rrp, rcols, rvals = A.data()
    assert np.array_equal(rp, rrp) and np.array_equal(cols, rcols)
    scale = np.repeat(np.maximum.reduceat(np.abs(rvals), rrp[:-1]), np.diff(rrp))
    assert np.max(np.abs(vals - rvals) / scale) <= 1e-14
    assert np.array_equal(_read(outd, "elasticity_b.bin", np.float64), b.get_local())

    up, vp = d2.TrialFunction(P1), d2.TestFunction(P1)
    form = d2.Constant(1.7) * d2.inner(d2.grad(up), d2.grad(vp)) * d2.dx
    A = d2.assemble(form)
    d2.assemble(form, tensor=A, add_values=True)
    for got, ref in zip(_matrix(outd, "add_values"), A.data()):
        assert np.array_equal(got, ref)

    msg = (outd / "error.txt").read_text()
    assert "Unable to assemble form" in msg and "Dim 0 of tensor does not match form" in msg
