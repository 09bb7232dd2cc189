"""dolfin_b200 -- a B200 (sm_100a) finite-element assembly engine with
DOLFIN 2019.1's assembly surface.

    from dolfin_b200 import *
    mesh = UnitCubeMesh(32, 32, 32)
    V = FunctionSpace(mesh, "Lagrange", 1)
    u, v = TrialFunction(V), TestFunction(V)
    kappa = Function(V, values)
    A = assemble(kappa*inner(grad(u), grad(v))*dx)     # device CSR
    rowptr, cols, vals = A.data()                      # as EigenMatrix.data()

Host structures (mesh, dofmap, sparsity pattern) follow DOLFIN's serial
numbering with parameters["reorder_dofs_serial"] = False; assembly runs in
hand-written CUDA kernels reached through the C ABI in include/dolfin_b200.h.
"""
from . import _capi
from .assembling import (SystemAssembler, assemble, assemble_action, assemble_local,
                         assemble_system)
from .io import File, XDMFFile
from .bcs import DirichletBC
from .cpp import (DofMap, FunctionSpace, Mesh, SparsityPattern, UnitCubeMesh, UnitSquareMesh,
                  VectorFunctionSpace, parameters)
from .function import Constant, Function
from .la import Matrix, Vector
from .ufl import (Identity, SpatialCoordinate, TestFunction, TrialFunction, div, dot, ds, dx, grad,
                  inner, nabla_grad, sym, tr, transpose)

__all__ = [
    "assemble", "assemble_system", "assemble_action", "assemble_local", "SystemAssembler", "File", "XDMFFile",
    "Mesh", "UnitCubeMesh",
    "UnitSquareMesh", "FunctionSpace", "VectorFunctionSpace", "DofMap", "SparsityPattern",
    "parameters", "Function", "Constant", "Matrix", "Vector", "TestFunction", "TrialFunction",
    "grad", "inner", "dot", "dx", "ds", "div", "sym", "tr", "transpose", "nabla_grad", "Identity",
    "DirichletBC", "SpatialCoordinate",
]


def kernel_launches():
    """Number of engine kernels launched by this process."""
    return _capi.kernel_launches()
