"""Differentiation of assembly with respect to a nodal (P1) coefficient.

``vjp_kappa`` runs the engine's adjoint kernels: given upstream gradients
gA (CSR-shaped, over the values of A = assemble(kappa*grad(u).grad(v)*dx))
and optionally gb (over b = assemble(kappa*f*v*dx)), it returns
dL/dkappa = sum gA * dA/dkappa + sum gb * db/dkappa -- the assembly of the
derivative form derivative(a, kappa) contracted with gA.  ``AssembleDiffusion``
wraps forward assembly and this adjoint in a torch.autograd.Function.
"""
from __future__ import annotations

import ctypes as C

import torch

from . import _capi
from ._capi import call
from .assembling import _PREC, _stream


def _p(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


def vjp_kappa(V, kappa, gA, f=None, gb=None, precision="fp64", scale=1.0, noalloc=False):
    """dL/dkappa (vertex field) for a = scale*kappa*grad(u).grad(v)*dx on V.

    noalloc=True uses db2_vjp_kappa_noalloc: the engine allocates no device
    memory during the call (fixed work array; see include/dolfin_b200.h)."""
    P = V.pattern()
    nv = V.mesh().num_vertices()
    kappa = kappa.contiguous().to(torch.float64)
    gA = gA.contiguous().to(torch.float64)
    if kappa.numel() != nv or gA.numel() != P.nnz():
        raise ValueError("kappa must be a vertex field and gA CSR-shaped")
    a = _capi.make_form(_capi.FORM_DIFFUSION, _capi.COEFF_P1_SCALED, (scale,))
    L = None
    if f is not None and gb is not None:
        L = _capi.make_form(_capi.FORM_LOAD, _capi.COEFF_P1_SCALED, (1.0,))
        f = f.contiguous().to(torch.float64)
        gb = gb.contiguous().to(torch.float64)
    dk = torch.empty(nv, dtype=torch.float64, device=kappa.device)
    call("db2_vjp_kappa_noalloc" if noalloc else "db2_vjp_kappa", P.handle, C.byref(a), _p(kappa), C.byref(L) if L is not None else None,
         _p(f), _p(gA), _p(gb), _PREC[precision], _p(dk), _stream())
    return dk


class AssembleDiffusion(torch.autograd.Function):
    """vals = assemble(kappa*inner(grad(u), grad(v))*dx).values on V, differentiable in kappa."""

    @staticmethod
    def forward(ctx, kappa, V, precision="fp64"):
        from .assembling import assemble
        from .function import Function
        from .cpp import FunctionSpace
        from .ufl import TestFunction, TrialFunction, dx, grad, inner
        W = V._p1_space if hasattr(V, "_p1_space") else None
        if W is None:
            W = FunctionSpace(V.mesh(), "Lagrange", 1)
            V._p1_space = W
        k = Function.__new__(Function)
        Function.__init__(k, W)
        k._x = kappa.detach().contiguous().to(torch.float64)
        u, v = TrialFunction(V), TestFunction(V)
        A = assemble(k * inner(grad(u), grad(v)) * dx, precision=precision)
        ctx.save_for_backward(kappa)
        ctx.V, ctx.precision = V, precision
        return A.values_tensor()

    @staticmethod
    def backward(ctx, gvals):
        (kappa,) = ctx.saved_tensors
        dk = vjp_kappa(ctx.V, kappa.detach(), gvals.contiguous(), precision=ctx.precision)
        return dk, None, None
