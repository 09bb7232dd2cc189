"""Differentiation of assembly with respect to a nodal (P1) coefficient.

``vjp_kappa`` runs the engine's adjoint kernels: given upstream gradients
gA (CSR-shaped, over the values of A = assemble(kappa*grad(u).grad(v)*dx))
and optionally gb (over b = assemble(kappa*f*v*dx)), it returns
dL/dkappa = sum gA * dA/dkappa + sum gb * db/dkappa -- the assembly of the
derivative form derivative(a, kappa) contracted with gA.  ``AssembleDiffusion``
wraps forward system assembly (A and b) and this adjoint in a
torch.autograd.Function.
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
        L = _capi.make_form(_capi.FORM_LOAD, _capi.COEFF_P1_KAPPA, (1.0,))
        f = f.contiguous().to(torch.float64)
        gb = gb.contiguous().to(torch.float64)
    dk = torch.empty(nv, dtype=torch.float64, device=kappa.device)
    call("db2_vjp_kappa_noalloc" if noalloc else "db2_vjp_kappa", P.handle, C.byref(a), _p(kappa), C.byref(L) if L is not None else None,
         _p(f), _p(gA), _p(gb), _PREC[precision], _p(dk), _stream())
    return dk


class AssembleDiffusion(torch.autograd.Function):
    """(A values, b) = assemble_system(kappa*inner(grad(u), grad(v))*dx, L) on
    V, differentiable in the P1 field kappa:

        L = kappa*f*v*dx   (weighted=True: b depends on kappa), or
        L = f*v*dx         (weighted=False: b does not),

    f a P1 vertex field (a tensor).  Backward runs the engine's adjoint:
    dL/dkappa = sum gA dA/dkappa + sum gb db/dkappa for the upstream
    gradients gA (over the CSR values) and gb (over b).

        vals, b = AssembleDiffusion.apply(kappa, V, f, True, "fp64")
    """

    @staticmethod
    def forward(ctx, kappa, V, f, weighted=True, precision="fp64"):
        from .assembling import SystemAssembler
        from .function import Function
        from .cpp import FunctionSpace
        from .ufl import TestFunction, TrialFunction, dx, grad, inner
        W = getattr(V, "_p1_space", None)
        if W is None:
            W = FunctionSpace(V.mesh(), "Lagrange", 1)
            V._p1_space = W
        kt = kappa.detach().contiguous().to(torch.float64)
        ft = f.detach().contiguous().to(torch.float64)
        k, fn = Function(W, kt), Function(W, ft)  # device tensors, not copied
        u, v = TrialFunction(V), TestFunction(V)
        L = (k * fn * v * dx) if weighted else (fn * v * dx)
        A, b = SystemAssembler(k * inner(grad(u), grad(v)) * dx, L, precision=precision).assemble()
        ctx.save_for_backward(kt, ft)
        ctx.V, ctx.precision, ctx.weighted = V, precision, weighted
        return A.values_tensor(), b.tensor()

    @staticmethod
    def backward(ctx, gvals, gb):
        kt, ft = ctx.saved_tensors
        if gvals is None:
            gvals = torch.zeros(ctx.V.pattern().nnz(), dtype=torch.float64, device=kt.device)
        use_b = ctx.weighted and gb is not None
        dk = vjp_kappa(ctx.V, kt, gvals.contiguous(), f=ft if use_b else None,
                       gb=gb.contiguous() if use_b else None, precision=ctx.precision)
        return dk, None, None, None, None
