"""Meshes, function spaces and sparsity patterns: thin owners of C-ABI handles.

Mirrors the parts of DOLFIN's Python surface the assembly path touches:
``Mesh`` / ``UnitCubeMesh`` / ``UnitSquareMesh`` (dolfin/mesh, dolfin/generation),
``FunctionSpace`` / ``VectorFunctionSpace`` with their ``DofMap``
(dolfin/function/FunctionSpace.h, dolfin/fem/DofMap.h) and the sparsity
pattern (dolfin/la/SparsityPattern.h).
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import _capi
from ._capi import call

parameters = {
    # DOLFIN's default is True (RCM reordering); the engine reproduces the
    # natural UFC numbering, which is what the reference's own assembly bench
    # and known-answer tests use (bench/fem/assembly/cpp/main.cpp:58).
    "reorder_dofs_serial": False,
    "linear_algebra_backend": "Eigen",
}


def _ptr(a):
    return C.c_void_p(a.ctypes.data) if a is not None else None


class _Handle:
    _destroy = None

    def __init__(self, h):
        self._h = h

    @property
    def handle(self):
        return self._h

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and self._destroy and _capi._lib is not None:
            try:
                getattr(_capi.lib(), self._destroy)(h)
            except Exception:
                pass
            self._h = None


class Mesh(_Handle):
    """Simplicial mesh (triangles or tetrahedra); cell vertex lists sorted."""
    _destroy = "db2_mesh_destroy"

    def __init__(self, coordinates=None, cells=None, _handle=None):
        if _handle is None and (isinstance(coordinates, (str, bytes)) or hasattr(coordinates, "__fspath__")):
            # Mesh("mesh.xml"): DOLFIN XML (dolfin/io/XMLMesh.cpp);
            # Mesh("mesh.xdmf"): XDMF with inline data (dolfin/io/XDMFFile.cpp)
            h = C.c_void_p()
            name = os.fsencode(coordinates)
            call("db2_mesh_read_xdmf" if name.endswith(b".xdmf") else "db2_mesh_read_xml", name, C.byref(h))
            _handle = h
        if _handle is None:
            x = np.ascontiguousarray(coordinates, np.float64)
            c = np.ascontiguousarray(cells, np.uint32)
            tdim = c.shape[1] - 1
            if x.ndim != 2 or x.shape[1] != tdim:
                raise ValueError("coordinates must be (nv, tdim) with gdim == tdim")
            h = C.c_void_p()
            call("db2_mesh_create", tdim, x.shape[0], _ptr(x), c.shape[0], _ptr(c), C.byref(h))
            _handle = h
        super().__init__(_handle)
        tdim, nv, nc = C.c_int(), C.c_int64(), C.c_int64()
        call("db2_mesh_info", self._h, C.byref(tdim), C.byref(nv), C.byref(nc))
        self._tdim, self._nv, self._nc = tdim.value, nv.value, nc.value

    def geometry_dim(self):
        return self._tdim

    def topology_dim(self):
        return self._tdim

    def num_vertices(self):
        return self._nv

    def num_cells(self):
        return self._nc

    def num_edges(self):
        ne = C.c_int64()
        call("db2_mesh_num_edges", self._h, C.byref(ne))
        return ne.value

    def num_exterior_facets(self):
        n = C.c_int64()
        call("db2_mesh_num_exterior_facets", self._h, C.byref(n))
        return n.value

    def exterior_facets(self):
        """(cell, local facet) of each exterior facet, in facet-number order."""
        n = self.num_exterior_facets()
        cell = np.empty(n, np.uint32)
        local = np.empty(n, np.int32)
        call("db2_mesh_exterior_facets", self._h, _ptr(cell), _ptr(local))
        return cell, local

    def coordinates(self):
        x = np.empty((self._nv, self._tdim), np.float64)
        call("db2_mesh_copy", self._h, _ptr(x), None)
        return x

    def cells(self):
        c = np.empty((self._nc, self._tdim + 1), np.uint32)
        call("db2_mesh_copy", self._h, None, _ptr(c))
        return c

    def set_coordinates(self, x):
        x = np.ascontiguousarray(x, np.float64)
        if x.shape != (self._nv, self._tdim):
            raise ValueError("coordinate array has the wrong shape")
        call("db2_mesh_set_coordinates", self._h, _ptr(x))

    def ufl_cell(self):
        return "tetrahedron" if self._tdim == 3 else "triangle"


def UnitCubeMesh(nx, ny, nz):
    """dolfin.UnitCubeMesh: 6 tetrahedra per cube (BoxMesh::build_tet)."""
    h = C.c_void_p()
    call("db2_mesh_unit_cube", int(nx), int(ny), int(nz), C.byref(h))
    return Mesh(_handle=h)


_DIAG = {"right": 0, "left": 1, "right/left": 2, "left/right": 3}


def UnitSquareMesh(nx, ny, diagonal="right"):
    """dolfin.UnitSquareMesh (RectangleMesh::build_tri)."""
    if diagonal not in _DIAG:
        raise ValueError(f"Unknown mesh diagonal definition: {diagonal}")
    h = C.c_void_p()
    call("db2_mesh_unit_square", int(nx), int(ny), _DIAG[diagonal], C.byref(h))
    return Mesh(_handle=h)


class DofMap:
    """dolfin.DofMap view of a function space (natural UFC numbering)."""

    def __init__(self, V):
        self._V = V
        self._cd = None

    def _all(self):
        if self._cd is None:
            out = np.empty((self._V.mesh().num_cells(), self._V._ndofs_cell), np.int32)
            call("db2_space_cell_dofs", self._V.handle, _ptr(out))
            self._cd = out
        return self._cd

    def cell_dofs(self, cell_index):
        return self._all()[cell_index].copy()

    def cell_dofs_all(self):
        return self._all()

    def global_dimension(self):
        return self._V.dim()

    def num_element_dofs(self, cell_index=0):
        return self._V._ndofs_cell

    def block_size(self):
        # block size is 1 without reordering (DofMapBuilder.cpp:97-99)
        return 1


_FAMILIES = {"Lagrange", "CG", "P"}


class FunctionSpace(_Handle):
    """Continuous Lagrange space of degree 1 or 2, scalar or vector valued."""
    _destroy = "db2_space_destroy"

    def __init__(self, mesh, family="Lagrange", degree=1, value_size=1):
        if family not in _FAMILIES:
            raise NotImplementedError(f"family {family!r}: only continuous Lagrange is provided")
        # reorder_dofs_serial = True: the reference's reverse Cuthill-McKee
        # numbering (dof_ordering_library "Boost"), dofs bs*node + c
        self._reordered = bool(parameters.get("reorder_dofs_serial", False))
        h = C.c_void_p()
        call("db2_space_create_reordered" if self._reordered else "db2_space_create",
             mesh.handle, int(degree), int(value_size), C.byref(h))
        super().__init__(h)
        self._mesh = mesh
        self._degree = int(degree)
        self._vs = int(value_size)
        k, n = C.c_int(), C.c_int64()
        call("db2_space_info", self._h, C.byref(k), C.byref(n))
        self._ndofs_cell, self._dim = k.value, n.value
        self._dofmap = DofMap(self)
        self._patterns = {}

    def mesh(self):
        return self._mesh

    def dim(self):
        return self._dim

    def reordered(self):
        return self._reordered

    def node_numbers(self):
        """Number of each natural node (vertex index, then nv + edge index)."""
        if getattr(self, "_node_new", None) is None:
            out = np.empty(self._dim // self._vs, np.int32)
            call("db2_space_node_numbers", self._h, _ptr(out))
            self._node_new = out
        return self._node_new

    def node_dofs(self, comp, nodes):
        """Dofs of component `comp` at natural nodes `nodes`."""
        nodes = np.asarray(nodes, np.int64)
        if self._reordered:
            return self._vs * self.node_numbers()[nodes].astype(np.int64) + comp
        return comp * (self._dim // self._vs) + nodes

    def degree(self):
        return self._degree

    def value_size(self):
        return self._vs

    def num_sub_spaces(self):
        return self._vs if self._vs > 1 else 0

    def dofmap(self):
        return self._dofmap

    def pattern(self, keep_diagonal=False):
        key = bool(keep_diagonal)
        if key not in self._patterns:
            self._patterns[key] = SparsityPattern(self, keep_diagonal)
        return self._patterns[key]

    def __eq__(self, other):
        return self is other

    def __hash__(self):
        return id(self)


def VectorFunctionSpace(mesh, family="Lagrange", degree=1, dim=None):
    return FunctionSpace(mesh, family, degree, value_size=dim or mesh.geometry_dim())


class SparsityPattern(_Handle):
    """Sorted CSR pattern of a form on V x V plus the engine's assembly plan."""
    _destroy = "db2_pattern_destroy"

    def __init__(self, V, keep_diagonal=False):
        h = C.c_void_p()
        call("db2_pattern_create", V.handle, int(bool(keep_diagonal)), C.byref(h))
        super().__init__(h)
        self.V = V
        nr, nnz = C.c_int64(), C.c_int64()
        call("db2_pattern_info", self._h, C.byref(nr), C.byref(nnz))
        self.nrows, self._nnz = nr.value, nnz.value
        self._dev = None

    def nnz(self):
        return self._nnz

    def csr_host(self):
        rp = np.empty(self.nrows + 1, np.int32)
        cols = np.empty(self._nnz, np.int32)
        call("db2_pattern_csr_host", self._h, _ptr(rp), _ptr(cols))
        return rp, cols

    def csr_device(self):
        """(rowptr, cols) as torch int32 tensors viewing the pattern's device arrays."""
        if self._dev is None:
            import torch
            rp, cols = C.c_void_p(), C.c_void_p()
            call("db2_pattern_csr_device", self._h, C.byref(rp), C.byref(cols))
            self._dev = (_wrap_device(rp.value, self.nrows + 1, torch.int32, self),
                         _wrap_device(cols.value, self._nnz, torch.int32, self))
        return self._dev

    def plan(self):
        nn, ninc, kp, nt = C.c_int64(), C.c_int64(), C.c_int(), C.c_int64()
        ng, ntyp = C.c_int64(), C.c_int64()
        call("db2_pattern_plan_info", self._h, C.byref(nn), C.byref(ninc), C.byref(kp), C.byref(nt),
             C.byref(ng), C.byref(ntyp))
        nn, ninc, kp, nt = nn.value, ninc.value, kp.value, nt.value
        self.ngroups, self.ntypes = ng.value, ntyp.value
        node_rowptr = np.empty(nn + 1, np.int32)
        rp = node_rowptr
        call("db2_pattern_plan_copy", self._h, _ptr(rp), None, None, None, None, None)
        node_cols = np.empty(int(rp[-1]), np.int32)
        inc_ptr = np.empty(nn + 1, np.uint32)
        inc = np.empty(ninc, np.uint32)
        pos = np.empty(ninc * kp, np.uint8)
        tiles = np.empty((nt, 4), np.int32)
        call("db2_pattern_plan_copy", self._h, None, _ptr(node_cols), _ptr(inc_ptr), _ptr(inc),
             _ptr(pos), _ptr(tiles))
        return dict(node_rowptr=node_rowptr, node_cols=node_cols, inc_ptr=inc_ptr, inc=inc,
                    pos=pos.reshape(ninc, kp), tiles=tiles, kp=kp)

    def inc_ptr(self):
        """Node -> incidence offsets alone (the work weights of the rows)."""
        nn, ninc, kp, nt = C.c_int64(), C.c_int64(), C.c_int(), C.c_int64()
        call("db2_pattern_plan_info", self._h, C.byref(nn), C.byref(ninc), C.byref(kp), C.byref(nt),
             None, None)
        out = np.empty(nn.value + 1, np.uint32)
        call("db2_pattern_plan_copy", self._h, None, None, _ptr(out), None, None, None)
        return out

    def retile(self, tile_threads, seg_cap_bytes):
        """Launch shape of the assembly kernel (see db2_pattern_retile)."""
        call("db2_pattern_retile", self._h, int(tile_threads), int(seg_cap_bytes))

    def set_row_range(self, node_begin, node_end):
        """Assemble only the rows of nodes [node_begin, node_end) (a rank's
        share of a row-partitioned assembly; see db2_pattern_set_row_range)."""
        call("db2_pattern_set_row_range", self._h, int(node_begin), int(node_end))
        self._block = False

    def set_row_block(self, node_begin, node_end):
        """As set_row_range, with the tensors holding the row block alone
        (a rank's own rows; see db2_pattern_set_row_block)."""
        call("db2_pattern_set_row_block", self._h, int(node_begin), int(node_end))
        self._block = True

    def holds_row_block(self):
        return getattr(self, "_block", False)

    def row_block_info(self):
        """(rows, nonzeros) of the current row block."""
        nr, nz = C.c_int64(), C.c_int64()
        call("db2_pattern_row_block_info", self._h, C.byref(nr), C.byref(nz))
        return int(nr.value), int(nz.value)

    def row_block_csr_host(self):
        """The row block's CSR: row pointers from 0 and global columns."""
        nr, nz = self.row_block_info()
        rp = np.empty(nr + 1, np.int32)
        cols = np.empty(nz, np.int32)
        call("db2_pattern_row_block_csr_host", self._h, _ptr(rp), _ptr(cols))
        return rp, cols


def _wrap_device(ptr, n, dtype, owner):
    """Zero-copy torch view of device memory owned by `owner` (kept alive)."""
    import torch

    class _Holder:
        def __init__(self, p, nbytes):
            self.__cuda_array_interface__ = {
                "shape": (n,), "typestr": {torch.int32: "<i4", torch.float64: "<f8"}[dtype],
                "data": (p, False), "version": 3, "strides": None}
            self.owner = owner

    t = torch.as_tensor(_Holder(ptr, n), device="cuda")
    return t
