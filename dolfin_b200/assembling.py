"""assemble(), assemble_system(), SystemAssembler -- the drop-in for
python/dolfin/fem/assembling.py (assemble :79-220, assemble_system :322-384,
_create_tensor :401-428), running the engine's CUDA kernels.

Keyword arguments keep DOLFIN's meaning: add_values (accumulate into an
existing tensor), finalize_tensor (no-op: device values are final when the
stream reaches them), keep_diagonal (pattern with the diagonal; the cell
pattern of a square Lagrange form already contains it), backend (only the
default).  The extra keyword ``precision`` selects the contraction
arithmetic ("fp64" or "fp32").
"""
from __future__ import annotations

import ctypes as C

from . import _capi
from ._capi import call
from .la import Matrix, Vector
from .ufl import Form, recognise

_PREC = {"fp64": _capi.FP64, "fp32": _capi.FP32_CONTRACT, None: _capi.FP64}


def _stream():
    import torch
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def _ptr(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


def _coeff_ptr(rec):
    if rec.function is None:
        return None
    f = rec.function
    if f.function_space().mesh() is not rec.V.mesh():
        raise ValueError("coefficient and form live on different meshes")
    return _ptr(f.tensor())


def _check_tensor_dims(tensor, rec):
    # AssemblerBase::init_global_tensor, dolfin/fem/AssemblerBase.cpp:182-191
    if tensor.size(0) != rec.V.dim():
        raise RuntimeError("*** Error: Unable to assemble form. Reason: Dim 0 of tensor does not match form.")


def assemble(form, tensor=None, form_compiler_parameters=None, add_values=False,
             finalize_tensor=True, keep_diagonal=False, backend=None, precision="fp64"):
    """Assemble a bilinear or linear form on the GPU (dolfin.assemble)."""
    if backend is not None:
        raise NotImplementedError("only the default backend (device CSR) is provided")
    if not isinstance(form, Form):
        raise TypeError("expected a Form")
    rec = recognise(form)
    prec = _PREC[precision]
    if rec.kind in (_capi.FORM_DIFFUSION, _capi.FORM_ELASTICITY):
        A = tensor if tensor is not None else Matrix()
        if A.empty():
            A.init(rec.V.pattern(keep_diagonal))
        else:
            _check_tensor_dims(A, rec)
            if A.pattern.V is not rec.V:
                raise RuntimeError("*** Error: tensor pattern belongs to another function space")
        call("db2_assemble_matrix", A.pattern.handle, C.byref(rec.c_form()), _coeff_ptr(rec), prec,
             _ptr(A.values_tensor()), int(bool(add_values)), _stream())
        return A
    b = tensor if tensor is not None else Vector(n=rec.V.dim())
    if b.size() != rec.V.dim():
        raise RuntimeError("*** Error: Unable to assemble form. Reason: Dim 0 of tensor does not match form.")
    call("db2_assemble_vector", rec.V.pattern(keep_diagonal).handle, C.byref(rec.c_form()),
         _coeff_ptr(rec), _ptr(b.tensor()), int(bool(add_values)), _stream())
    return b


class SystemAssembler:
    """SystemAssembler(a, L, bcs): A and b in one pass
    (dolfin/fem/SystemAssembler.cpp:138-301, cell_wise_assembly :303-492)."""

    def __init__(self, a, L, bcs=None, precision="fp64"):
        self.ra, self.rL = recognise(a), recognise(L)
        if self.ra.V is not self.rL.V:
            raise RuntimeError("a and L must share the function space")
        self.bcs = [] if bcs is None else (bcs if isinstance(bcs, (list, tuple)) else [bcs])
        self.prec = _PREC[precision]
        self.keep_diagonal = False

    def assemble(self, A=None, b=None):
        V = self.ra.V
        if A is None and b is None:
            A, b = Matrix(), Vector(n=V.dim())
        if A is not None and A.empty():
            A.init(V.pattern(self.keep_diagonal))
        if b is None:
            b = Vector(n=V.dim())
        if A is None:
            return self._vector_only(b)
        if self.bcs:
            flags, vals = _bc_arrays(V, self.bcs)
            call("db2_assemble_system_bc", A.pattern.handle, C.byref(self.ra.c_form()),
                 _coeff_ptr(self.ra), C.byref(self.rL.c_form()), _coeff_ptr(self.rL), _ptr(flags),
                 _ptr(vals), self.prec, _ptr(A.values_tensor()), _ptr(b.tensor()), _stream())
        else:
            call("db2_assemble_system", A.pattern.handle, C.byref(self.ra.c_form()),
                 _coeff_ptr(self.ra), C.byref(self.rL.c_form()), _coeff_ptr(self.rL), self.prec,
                 _ptr(A.values_tensor()), _ptr(b.tensor()), _stream())
        return A, b

    def _vector_only(self, b):
        call("db2_assemble_vector", self.rL.V.pattern(False).handle, C.byref(self.rL.c_form()),
             _coeff_ptr(self.rL), _ptr(b.tensor()), 0, _stream())
        return b


def assemble_system(A_form, b_form, bcs=None, x0=None, form_compiler_parameters=None,
                    add_values=False, finalize_tensor=True, keep_diagonal=False, A_tensor=None,
                    b_tensor=None, backend=None, precision="fp64"):
    """dolfin.assemble_system (python/dolfin/fem/assembling.py:322-384)."""
    if x0 is not None:
        raise NotImplementedError("x0 (incremental boundary values) is not provided")
    if add_values:
        raise NotImplementedError("add_values with assemble_system is not provided")
    S = SystemAssembler(A_form, b_form, bcs, precision)
    S.keep_diagonal = keep_diagonal
    A = A_tensor if A_tensor is not None else Matrix()
    b = b_tensor if b_tensor is not None else Vector(n=S.ra.V.dim())
    return S.assemble(A, b)


def assemble_action(a, x, y=None, precision="fp64"):
    """Matrix-free y = A(a) x without forming A (replaces assemble + GenericMatrix::mult)."""
    rec = recognise(a)
    xt = x.tensor() if hasattr(x, "tensor") else x
    if xt.numel() != rec.V.dim():
        raise RuntimeError("x has the wrong size")
    if y is None:
        y = Vector(n=rec.V.dim())
    call("db2_apply", rec.V.pattern(False).handle, C.byref(rec.c_form()), _coeff_ptr(rec),
         _PREC[precision], _ptr(xt.contiguous()), _ptr(y.tensor()), _stream())
    return y


def _bc_arrays(V, bcs):
    import torch
    flags = torch.zeros(V.dim(), dtype=torch.uint8, device="cuda")
    vals = torch.zeros(V.dim(), dtype=torch.float64, device="cuda")
    for bc in bcs:
        dofs, values = bc.dofs_and_values()
        d = torch.as_tensor(dofs, dtype=torch.int64, device="cuda")
        flags[d] = 1
        vals[d] = torch.as_tensor(values, dtype=torch.float64, device="cuda")
    return flags, vals
