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
from .ufl import Form, Recognised, recognise_functional, recognise_parts

# "fp32_tc" (the matrix-free action of P2 diffusion only): the FP32
# contraction on the tensor cores
_PREC = {"fp64": _capi.FP64, "fp32": _capi.FP32_CONTRACT, "fp32_tc": _capi.FP32_TENSOR_CORE,
         None: _capi.FP64}


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
    return _ptr(f.vertex_tensor())


def _parts(form):
    """recognise_parts(form), computed once per Form object (forms and
    Constants are immutable; Functions are read through their device
    tensors at each call), so repeated assemblies spend no host time on
    recognition."""
    parts = getattr(form, "_db2_parts", None)
    if parts is None:
        parts = recognise_parts(form)
        form._db2_parts = parts
    return parts


def _whole(P):
    if P.holds_row_block():
        raise RuntimeError("the pattern is set to a row block (shard.RowBlock holds its tensors); "
                           "set_row_range(0, nnodes) restores whole-matrix assembly")


def _check_tensor_dims(tensor, rec):
    # AssemblerBase::init_global_tensor, dolfin/fem/AssemblerBase.cpp:182-191
    if tensor.size(0) != rec.V.dim():
        raise RuntimeError("*** Error: Unable to assemble form. Reason: Dim 0 of tensor does not match form.")


def assemble(form, tensor=None, form_compiler_parameters=None, add_values=False,
             finalize_tensor=True, keep_diagonal=False, backend=None, precision="fp64"):
    """Assemble a form on the GPU (dolfin.assemble): a Matrix for bilinear, a
    Vector for linear forms, a float for functionals.  dx terms run the cell
    kernels, ds terms then add the exterior-facet contributions (the
    reference's cell loop, then exterior-facet loop, Assembler.cpp:52-103)."""
    if backend is not None:
        raise NotImplementedError("only the default backend (device CSR) is provided")
    if not isinstance(form, Form):
        raise TypeError("expected a Form")
    if form.rank() == 0:
        return _assemble_scalar(form)
    cell, facet = _parts(form)
    rec = cell or facet
    prec = _PREC[precision]
    parts = [r for r in (cell, facet) if r is not None]
    if form.rank() == 2:
        A = tensor if tensor is not None else Matrix()
        if A.empty():
            A.init(rec.V.pattern(keep_diagonal))
        else:
            _check_tensor_dims(A, rec)
            if A.pattern.V is not rec.V:
                raise RuntimeError("*** Error: tensor pattern belongs to another function space")
        _whole(A.pattern)
        for i, r in enumerate(parts):
            call("db2_assemble_matrix", A.pattern.handle, C.byref(r.c_form()), _coeff_ptr(r), prec,
                 _ptr(A.values_tensor()), int(bool(add_values) or i > 0), _stream())
        return A
    if cell is not None and cell.pair is not None:
        raise NotImplementedError("kappa*f*v*dx is assembled with its bilinear form: use "
                                  "assemble_system / SystemAssembler")
    b = tensor if tensor is not None else Vector(n=rec.V.dim())
    if b.size() != rec.V.dim():
        raise RuntimeError("*** Error: Unable to assemble form. Reason: Dim 0 of tensor does not match form.")
    _whole(rec.V.pattern(keep_diagonal))
    for i, r in enumerate(parts):
        call("db2_assemble_vector", rec.V.pattern(keep_diagonal).handle, C.byref(r.c_form()),
             _coeff_ptr(r), _ptr(b.tensor()), int(bool(add_values) or i > 0), _stream())
    return b


def assemble_local(form, cell):
    """dolfin.assemble_local (LocalAssembler::assemble,
    dolfin/fem/LocalAssembler.cpp:39-98): the element tensor of `cell` in its
    local dof order (cell integral + the cell's exterior-facet integrals), as
    a numpy array (n, n) or (n,).  `cell` may also be an array of cell
    indices: then the tensors of all of them, (m, n, n) or (m, n), computed
    in one launch."""
    import numpy as np
    import torch
    if not isinstance(form, Form):
        raise TypeError("expected a Form")
    if form.rank() == 0:
        raise NotImplementedError("assemble_local of a functional is not provided")
    cell_rec, facet_rec = _parts(form)
    rec = cell_rec or facet_rec
    V = rec.V
    idx = np.atleast_1d(np.asarray(cell, dtype=np.int64))
    nc = V.mesh().num_cells()
    if idx.size and (idx.min() < 0 or idx.max() >= nc):
        raise IndexError(f"cell index out of range (mesh has {nc} cells)")
    cells = torch.as_tensor(idx.astype(np.uint32).view(np.int32), device="cuda")
    n = V._ndofs_cell
    shape = (idx.size, n, n) if form.rank() == 2 else (idx.size, n)
    out = torch.empty(shape, dtype=torch.float64, device="cuda")
    call("db2_assemble_local", V.handle,
         C.byref(cell_rec.c_form()) if cell_rec is not None else None,
         _coeff_ptr(cell_rec) if cell_rec is not None else None,
         C.byref(facet_rec.c_form()) if facet_rec is not None else None,
         _coeff_ptr(facet_rec) if facet_rec is not None else None,
         int(idx.size), _ptr(cells), _ptr(out), _stream())
    res = out.cpu().numpy()
    return res[0] if np.ndim(cell) == 0 else res


def _assemble_scalar(form):
    """double assemble(const Form&) (dolfin/fem/assemble.h:66): the sum of
    the dx and ds parts, each reduced on the device in a fixed order."""
    import torch
    total = 0.0
    for kind, mesh, coeff, func, const in recognise_functional(form):
        w = None
        if func is not None:
            if func.function_space().mesh() is not mesh:
                raise ValueError("coefficient and form live on different meshes")
            w = _ptr(func.vertex_tensor())
        out = torch.empty(1, dtype=torch.float64, device="cuda")
        call("db2_assemble_scalar", mesh.handle, C.byref(_capi.make_form(kind, coeff, const)), w,
             _ptr(out), _stream())
        total += float(out.item())
    return total


class SystemAssembler:
    """SystemAssembler(a, L, bcs): A and b in one pass
    (dolfin/fem/SystemAssembler.cpp:138-301, cell_wise_assembly :303-492)."""

    def __init__(self, a, L, bcs=None, precision="fp64"):
        self.ra, self.ra_ds = _parts(a)
        self.rL, self.rL_ds = _parts(L)
        if self.ra is None:
            raise NotImplementedError("the bilinear form needs a cell (dx) part")
        if self.rL is None:
            # L has only ds terms: the cell pass assembles a zero load
            self.rL = Recognised(_capi.FORM_LOAD, self.ra.V, _capi.COEFF_CONSTANT, None,
                                 (0.0, 0.0, 0.0))
        if self.ra.V is not self.rL.V:
            raise RuntimeError("a and L must share the function space")
        if self.rL.pair is not None:
            # kappa*f*v*dx: kappa is the bilinear form's P1 coefficient
            self.rL = self.rL.with_kappa(self.ra.function)
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
        _whole(A.pattern)
        self.assemble_into(A.pattern, A.values_tensor(), b.tensor())
        return A, b

    def assemble_into(self, P, vt, bt):
        """Assemble A and b into the device tensors vt (CSR values of pattern
        P, or its row block) and bt."""
        if self.bcs:
            flags, vals = _bc_arrays(self.ra.V, self.bcs)
            call("db2_assemble_system_bc", P.handle, C.byref(self.ra.c_form()),
                 _coeff_ptr(self.ra), C.byref(self.rL.c_form()), _coeff_ptr(self.rL), _ptr(flags),
                 _ptr(vals), self.prec, _ptr(vt), _ptr(bt), _stream())
            if self.ra_ds is not None or self.rL_ds is not None:
                # exterior-facet terms with the same Dirichlet treatment
                fa = C.byref(self.ra_ds.c_form()) if self.ra_ds is not None else None
                fl = C.byref(self.rL_ds.c_form()) if self.rL_ds is not None else None
                call("db2_assemble_facets_bc", P.handle, fa,
                     _coeff_ptr(self.ra_ds) if self.ra_ds is not None else None, fl,
                     _coeff_ptr(self.rL_ds) if self.rL_ds is not None else None, _ptr(flags),
                     _ptr(vals), _ptr(vt), _ptr(bt), _stream())
        else:
            call("db2_assemble_system", P.handle, C.byref(self.ra.c_form()),
                 _coeff_ptr(self.ra), C.byref(self.rL.c_form()), _coeff_ptr(self.rL), self.prec,
                 _ptr(vt), _ptr(bt), _stream())
            if self.ra_ds is not None:
                call("db2_assemble_matrix", P.handle, C.byref(self.ra_ds.c_form()),
                     _coeff_ptr(self.ra_ds), self.prec, _ptr(vt), 1, _stream())
            if self.rL_ds is not None:
                call("db2_assemble_vector", P.handle, C.byref(self.rL_ds.c_form()),
                     _coeff_ptr(self.rL_ds), _ptr(bt), 1, _stream())

    def _vector_only(self, b):
        P = self.rL.V.pattern(False)
        call("db2_assemble_vector", P.handle, C.byref(self.rL.c_form()),
             _coeff_ptr(self.rL), _ptr(b.tensor()), 0, _stream())
        if self.rL_ds is not None:
            call("db2_assemble_vector", P.handle, C.byref(self.rL_ds.c_form()),
                 _coeff_ptr(self.rL_ds), _ptr(b.tensor()), 1, _stream())
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
    if "ds" in a.measures():
        raise NotImplementedError("matrix-free action of ds terms is not provided")
    rec = _parts(a)[0]
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
