"""ctypes wrapper of the CPU oracle (liboracle.so).

TEST INFRASTRUCTURE ONLY: the correctness checker of the CUDA engine and the
timed CPU baseline.  Only ``tests/``, ``__graft_entry__.smoke()`` and the
``cpu_baseline`` leg of ``bench.py`` import this module; the product package
``dolfin_b200`` never does.

The C++ behind it restates DOLFIN 2019.1's serial assembly path; each
function in ``oracle.cpp`` cites the reference file:line it follows.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

DIFFUSION, MASS, LOAD, ELASTICITY, DIV_P, GRADP_V, FUNCTIONAL = 1, 2, 3, 4, 5, 6, 7
FACET_MASS, FACET_LOAD, FACET_FUNCTIONAL = 8, 9, 10
COEFF_NONE, COEFF_CONST, COEFF_P1, COEFF_X0, COEFF_P1_TIMES_P1 = 0, 1, 2, 3, 4
CG, DG = 0, 1


class OrcForm(C.Structure):
    _fields_ = [
        ("kind", C.c_int), ("tdim", C.c_int), ("gdim", C.c_int),
        ("family0", C.c_int), ("degree0", C.c_int), ("vsize0", C.c_int),
        ("family1", C.c_int), ("degree1", C.c_int), ("vsize1", C.c_int),
        ("coeff", C.c_int), ("c", C.c_double * 3), ("mu", C.c_double), ("lmbda", C.c_double),
    ]


def build():
    """Compile liboracle.so with its Makefile (g++ only)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        L = C.CDLL(path)
        P = C.c_void_p
        i64, i32 = C.c_int64, C.c_int
        L.orc_box_mesh.argtypes = [i32, i32, i32, P, P]
        L.orc_rectangle_mesh.argtypes = [i32, i32, i32, P, P]
        L.orc_interval_mesh.argtypes = [i32, P, P]
        L.orc_edges.argtypes = [i32, i64, P, P, P]
        L.orc_edges.restype = i64
        L.orc_dofmap.argtypes = [i32, i32, i32, i32, i64, i64, P, P]
        L.orc_dofmap.restype = i64
        L.orc_ndofs_per_cell.argtypes = [i32, i32, i32, i32]
        L.orc_dofmap_reordered.argtypes = [i32, i32, i32, i64, i64, P, P, P]
        L.orc_dofmap_reordered.restype = i64
        L.orc_sparsity.argtypes = [i64, i64, i64, i32, P, i32, P, i32]
        L.orc_sparsity.restype = P
        L.orc_csr_nnz.argtypes = [P]
        L.orc_csr_nnz.restype = i64
        L.orc_csr_copy.argtypes = [P, P, P]
        L.orc_csr_free.argtypes = [P]
        L.orc_element_tensor.argtypes = [P, P, P, P, P]
        L.orc_assemble_matrix.argtypes = [P, i64, P, i64, P, P, P, P, P, i64, P, P, P, i32]
        L.orc_assemble_vector.argtypes = [P, i64, P, i64, P, P, P, P, i64, P, i32]
        L.orc_assemble_scalar.argtypes = [P, i64, P, i64, P, P]
        L.orc_assemble_scalar.restype = C.c_double
        L.orc_assemble_system.argtypes = [P, P, i64, P, i64, P, P, P, P, i64, P, P, i64, P, P, P, P]
        L.orc_assemble_system_ds.argtypes = [P, P, P, P, i64, P, i64, P, P, P, P, P, P, i64, P, P,
                                             i64, P, P, P, P]
        L.orc_exterior_facets.argtypes = [i32, i64, P, P, P]
        L.orc_exterior_facets.restype = i64
        L.orc_boundary_vertices.argtypes = [i32, i64, P, P]
        L.orc_boundary_vertices.restype = i64
        L.orc_vjp_diffusion.argtypes = [P, i64, P, i64, P, P, P, P, P, P, P, i32, P]
        L.orc_quadrature_monomial.argtypes = [i32, i32, i32, i32, i32]
        L.orc_quadrature_monomial.restype = C.c_double
        _LIB = L
    return _LIB


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def form(kind, tdim, degree0=1, vsize0=1, degree1=None, vsize1=None, family0=CG, family1=CG,
         coeff=COEFF_NONE, c=(0.0, 0.0, 0.0), mu=0.0, lmbda=0.0):
    f = OrcForm()
    f.kind, f.tdim, f.gdim = kind, tdim, tdim
    f.family0, f.degree0, f.vsize0 = family0, degree0, vsize0
    f.family1 = family1
    f.degree1 = degree0 if degree1 is None else degree1
    f.vsize1 = vsize0 if vsize1 is None else vsize1
    f.coeff = coeff
    for i in range(3):
        f.c[i] = float(c[i]) if i < len(c) else 0.0
    f.mu, f.lmbda = float(mu), float(lmbda)
    return f


@dataclass
class Mesh:
    tdim: int
    coords: np.ndarray   # (nv, gdim) float64
    cells: np.ndarray    # (nc, tdim+1) uint32, sorted vertices

    @property
    def nv(self):
        return self.coords.shape[0]

    @property
    def nc(self):
        return self.cells.shape[0]


def unit_cube_mesh(nx, ny, nz):
    nv = (nx + 1) * (ny + 1) * (nz + 1)
    coords = np.empty((nv, 3), np.float64)
    cells = np.empty((6 * nx * ny * nz, 4), np.uint32)
    assert lib().orc_box_mesh(nx, ny, nz, _p(coords), _p(cells)) == 0
    return Mesh(3, coords, cells)


def unit_square_mesh(nx, ny, diagonal="right"):
    d = {"right": 0, "left": 1, "right/left": 2, "left/right": 3}[diagonal]
    coords = np.empty(((nx + 1) * (ny + 1), 2), np.float64)
    cells = np.empty((2 * nx * ny, 3), np.uint32)
    assert lib().orc_rectangle_mesh(nx, ny, d, _p(coords), _p(cells)) == 0
    return Mesh(2, coords, cells)


def unit_interval_mesh(n):
    coords = np.empty((n + 1, 1), np.float64)
    cells = np.empty((n, 2), np.uint32)
    assert lib().orc_interval_mesh(n, _p(coords), _p(cells)) == 0
    return Mesh(1, coords, cells)


def edges(mesh):
    ne_per = {3: 6, 2: 3}[mesh.tdim]
    ce = np.empty((mesh.nc, ne_per), np.uint32)
    cells = np.ascontiguousarray(mesh.cells)
    ne = lib().orc_edges(mesh.tdim, mesh.nc, _p(cells), _p(ce), None)
    ev = np.empty((ne, 2), np.uint32)
    lib().orc_edges(mesh.tdim, mesh.nc, _p(cells), _p(ce), _p(ev))
    return ce, ev


def dofmap(mesh, degree, vsize=1, family=CG):
    k = lib().orc_ndofs_per_cell(family, degree, vsize, mesh.tdim)
    out = np.empty((mesh.nc, k), np.int32)
    cells = np.ascontiguousarray(mesh.cells)
    n = lib().orc_dofmap(family, degree, vsize, mesh.tdim, mesh.nv, mesh.nc, _p(cells), _p(out))
    return out, int(n)


def dofmap_reordered(mesh, degree, vsize=1):
    """reorder_dofs_serial = True (Boost RCM): (cell dofs, dimension, node_new)."""
    k = lib().orc_ndofs_per_cell(CG, degree, vsize, mesh.tdim)
    out = np.empty((mesh.nc, k), np.int32)
    cells = np.ascontiguousarray(mesh.cells)
    nn = (mesh.nv + (edges(mesh)[1].shape[0] if degree == 2 else 0))
    node_new = np.empty(nn, np.int32)
    n = lib().orc_dofmap_reordered(degree, vsize, mesh.tdim, mesh.nv, mesh.nc, _p(cells), _p(out),
                                   _p(node_new))
    return out, int(n), node_new


def sparsity(nrows, ncols, dofs0, dofs1, keep_diagonal=False):
    dofs0 = np.ascontiguousarray(dofs0, np.int32)
    dofs1 = np.ascontiguousarray(dofs1, np.int32)
    h = lib().orc_sparsity(nrows, ncols, dofs0.shape[0], dofs0.shape[1], _p(dofs0),
                           dofs1.shape[1], _p(dofs1), int(keep_diagonal))
    nnz = lib().orc_csr_nnz(h)
    rowptr = np.empty(nrows + 1, np.int32)
    cols = np.empty(nnz, np.int32)
    lib().orc_csr_copy(h, _p(rowptr), _p(cols))
    lib().orc_csr_free(h)
    return rowptr, cols


def element_tensor(f, coordinate_dofs, w=None, w2=None, size=None):
    xc = np.ascontiguousarray(coordinate_dofs, np.float64).ravel()
    w = None if w is None else np.ascontiguousarray(w, np.float64)
    w2 = None if w2 is None else np.ascontiguousarray(w2, np.float64)
    out = np.zeros(size, np.float64)
    assert lib().orc_element_tensor(C.byref(f), _p(xc), _p(w), _p(w2), _p(out)) == 0
    return out


def assemble_matrix(f, mesh, dofs0, dofs1, rowptr, cols, w=None, w2=None):
    vals = np.zeros(cols.shape[0], np.float64)
    coords = np.ascontiguousarray(mesh.coords, np.float64)
    cells = np.ascontiguousarray(mesh.cells, np.uint32)
    rc = lib().orc_assemble_matrix(C.byref(f), mesh.nv, _p(coords), mesh.nc, _p(cells),
                                   _p(np.ascontiguousarray(dofs0, np.int32)),
                                   _p(np.ascontiguousarray(dofs1, np.int32)),
                                   _p(w), _p(w2), rowptr.shape[0] - 1, _p(rowptr), _p(cols),
                                   _p(vals), 0)
    if rc != 0:
        raise RuntimeError(f"oracle assemble_matrix failed ({rc})")
    return vals


def assemble_vector(f, mesh, dofs0, n, w=None, w2=None):
    b = np.zeros(n, np.float64)
    coords = np.ascontiguousarray(mesh.coords, np.float64)
    cells = np.ascontiguousarray(mesh.cells, np.uint32)
    lib().orc_assemble_vector(C.byref(f), mesh.nv, _p(coords), mesh.nc, _p(cells),
                              _p(np.ascontiguousarray(dofs0, np.int32)), _p(w), _p(w2), n,
                              _p(b), 0)
    return b


def assemble_scalar(f, mesh, w=None):
    coords = np.ascontiguousarray(mesh.coords, np.float64)
    cells = np.ascontiguousarray(mesh.cells, np.uint32)
    return lib().orc_assemble_scalar(C.byref(f), mesh.nv, _p(coords), mesh.nc, _p(cells), _p(w))


def assemble_system(a, L, mesh, dofs, n, rowptr, cols, bc_dofs, bc_vals, wa=None, wL=None):
    vals = np.zeros(cols.shape[0], np.float64)
    b = np.zeros(n, np.float64)
    coords = np.ascontiguousarray(mesh.coords, np.float64)
    cells = np.ascontiguousarray(mesh.cells, np.uint32)
    bc_dofs = np.ascontiguousarray(bc_dofs, np.int32)
    bc_vals = np.ascontiguousarray(bc_vals, np.float64)
    rc = lib().orc_assemble_system(C.byref(a), C.byref(L), mesh.nv, _p(coords), mesh.nc,
                                   _p(cells), _p(np.ascontiguousarray(dofs, np.int32)), _p(wa),
                                   _p(wL), bc_dofs.shape[0], _p(bc_dofs), _p(bc_vals), n,
                                   _p(rowptr), _p(cols), _p(vals), _p(b))
    if rc != 0:
        raise RuntimeError(f"oracle assemble_system failed ({rc})")
    return vals, b


def assemble_system_ds(a, L, mesh, dofs, n, rowptr, cols, bc_dofs, bc_vals, wa=None, wL=None,
                       a_ds=None, L_ds=None, wa_ds=None, wL_ds=None):
    """SystemAssembler with exterior facet integrals a_ds / L_ds (or None)."""
    vals = np.zeros(cols.shape[0], np.float64)
    b = np.zeros(n, np.float64)
    coords = np.ascontiguousarray(mesh.coords, np.float64)
    cells = np.ascontiguousarray(mesh.cells, np.uint32)
    bc_dofs = np.ascontiguousarray(bc_dofs, np.int32)
    bc_vals = np.ascontiguousarray(bc_vals, np.float64)
    ref = lambda f: None if f is None else C.byref(f)
    rc = lib().orc_assemble_system_ds(C.byref(a), ref(a_ds), C.byref(L), ref(L_ds), mesh.nv,
                                      _p(coords), mesh.nc, _p(cells),
                                      _p(np.ascontiguousarray(dofs, np.int32)), _p(wa), _p(wa_ds),
                                      _p(wL), _p(wL_ds), bc_dofs.shape[0], _p(bc_dofs),
                                      _p(bc_vals), n, _p(rowptr), _p(cols), _p(vals), _p(b))
    if rc != 0:
        raise RuntimeError(f"oracle assemble_system_ds failed ({rc})")
    return vals, b


def exterior_facets(mesh):
    """(cell, local facet) of each exterior facet, in facet-number order."""
    cells = np.ascontiguousarray(mesh.cells, np.uint32)
    cap = mesh.nc * (mesh.tdim + 1)
    fc = np.empty(cap, np.uint32)
    fl = np.empty(cap, np.int32)
    m = lib().orc_exterior_facets(mesh.tdim, mesh.nc, _p(cells), _p(fc), _p(fl))
    return fc[:m].copy(), fl[:m].copy()


def boundary_vertices(mesh):
    coords = np.ascontiguousarray(mesh.coords, np.float64)
    out = np.empty(mesh.nv, np.int32)
    m = lib().orc_boundary_vertices(coords.shape[1], mesh.nv, _p(coords), _p(out))
    return out[:m].copy()


def vjp_diffusion(a, mesh, dofs, rowptr, cols, gA, f=None, gb=None, load_has_kappa=False):
    dk = np.zeros(mesh.nv, np.float64)
    coords = np.ascontiguousarray(mesh.coords, np.float64)
    cells = np.ascontiguousarray(mesh.cells, np.uint32)
    rc = lib().orc_vjp_diffusion(C.byref(a), mesh.nv, _p(coords), mesh.nc, _p(cells),
                                 _p(np.ascontiguousarray(dofs, np.int32)), _p(rowptr), _p(cols),
                                 _p(np.ascontiguousarray(gA, np.float64)),
                                 _p(None if f is None else np.ascontiguousarray(f, np.float64)),
                                 _p(None if gb is None else np.ascontiguousarray(gb, np.float64)),
                                 int(load_has_kappa), _p(dk))
    if rc != 0:
        raise RuntimeError(f"oracle vjp failed ({rc})")
    return dk


def quadrature_monomial(tdim, degree, a, b=0, c=0):
    return lib().orc_quadrature_monomial(tdim, degree, a, b, c)
