"""Runs one named assembly workload a few times (for profiling with ncu).

    python -m dolfin_b200.profile_case {elas|p2|p1} N [REPS] [action]

elas: vector P2 elasticity on UnitCubeMesh(N) jittered 0.15h (A and b);
p2 / p1: kappa*grad(u).grad(v) + f*v on P2 / P1 with P1 kappa, f.
With "action" the matrix-free y = A x is run REPS times instead (x seeded).
"""
import sys, os
import torch, numpy as np
import dolfin_b200 as d2
from dolfin_b200 import synthetic
kind = sys.argv[1]; n = int(sys.argv[2]); reps = int(sys.argv[3]) if len(sys.argv) > 3 else 3
mesh = d2.UnitCubeMesh(n, n, n)
if kind == "elas":
    mesh.set_coordinates(synthetic.jitter_interior(mesh.coordinates(), n, 0.15, 1))
    V = d2.VectorFunctionSpace(mesh, "Lagrange", 2)
    u, v = d2.TrialFunction(V), d2.TestFunction(V)
    mu, lm = d2.Constant(1/2.6), d2.Constant(0.3/(1.3*0.4))
    eps = lambda w: d2.sym(d2.grad(w))
    a = d2.inner(2*mu*eps(u) + lm*d2.tr(eps(u))*d2.Identity(3), eps(v))*d2.dx
    L = d2.inner(d2.Constant((0.0, 0.0, -1.0)), v)*d2.dx
else:
    deg = 2 if kind == "p2" else 1
    V = d2.FunctionSpace(mesh, "Lagrange", deg)
    W = d2.FunctionSpace(mesh, "Lagrange", 1)
    kappa = d2.Function(W, synthetic.uniform_field(mesh.num_vertices(), 0.5, 2, 1))
    f = d2.Function(W, synthetic.uniform_field(mesh.num_vertices(), -1, 1, 2))
    u, v = d2.TrialFunction(V), d2.TestFunction(V)
    a = kappa*d2.inner(d2.grad(u), d2.grad(v))*d2.dx
    L = f*v*d2.dx
if len(sys.argv) > 4 and sys.argv[4] == "action":
    x = torch.randn(V.dim(), dtype=torch.float64, device="cuda",
                    generator=torch.Generator("cuda").manual_seed(3))
    y = d2.Vector(torch.empty_like(x))
    for _ in range(reps):
        d2.assemble_action(a, d2.Vector(x), y)
    torch.cuda.synchronize()
    print(kind, n, "cells", mesh.num_cells(), "action |y|", float(y.tensor().norm()))
    sys.exit(0)
S = d2.SystemAssembler(a, L)
A, b = d2.Matrix(), d2.Vector(n=V.dim())
for _ in range(reps):
    S.assemble(A, b)
torch.cuda.synchronize()
print(kind, n, "cells", mesh.num_cells(), "nnz", A.nnz(), "norm", A.norm())
