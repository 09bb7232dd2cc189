"""File -- DOLFIN XML input/output of meshes and vectors (dolfin.File with
the .xml suffix: dolfin/io/File.cpp, XMLFile.cpp, XMLMesh.cpp, XMLVector.cpp).

    File("mesh.xml") << mesh        File("b.xml") << b
    mesh = Mesh("mesh.xml")         File("b.xml") >> b

XDMFFile -- XDMF meshes with inline (ASCII) data (dolfin/io/XDMFFile.cpp):

    with XDMFFile("mesh.xdmf") as f: f.write(mesh)      # or f.write(u), u P1
    mesh = Mesh("mesh.xdmf");  XDMFFile("mesh.xdmf").read(mesh)

The files are read and written by the engine library (C++); vectors are
copied between device and host around the call.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import _capi
from ._capi import call


class File:
    def __init__(self, filename, mode="w"):
        name = os.fspath(filename)
        if not name.endswith(".xml"):
            raise NotImplementedError("only DOLFIN XML files (.xml) are provided")
        self.name = name

    def __lshift__(self, obj):
        from .cpp import Mesh
        from .la import Vector
        if isinstance(obj, Mesh):
            call("db2_mesh_write_xml", obj.handle, os.fsencode(self.name))
        elif isinstance(obj, Vector):
            x = np.ascontiguousarray(obj.get_local(), np.float64)
            call("db2_vector_write_xml", os.fsencode(self.name), x.shape[0],
                 C.c_void_p(x.ctypes.data))
        else:
            raise NotImplementedError(f"File << {type(obj).__name__} is not provided")
        return self

    def __rshift__(self, obj):
        import torch
        from .la import Vector
        if not isinstance(obj, Vector):
            raise NotImplementedError("File >> is provided for Vector; read meshes with Mesh(filename)")
        n = C.c_int64(0)
        call("db2_vector_read_xml", os.fsencode(self.name), C.byref(n), None)
        x = np.empty(n.value, np.float64)
        call("db2_vector_read_xml", os.fsencode(self.name), C.byref(n), C.c_void_p(x.ctypes.data))
        t = torch.as_tensor(x)
        obj._x = t.to("cuda") if torch.cuda.is_available() else t
        return self


class XDMFFile:
    """dolfin.XDMFFile for meshes and P1 vertex fields with ASCII encoding.

    ``XDMFFile.Encoding.HDF5`` (DOLFIN's default) needs HDF5, which is not
    part of this build: writing with it raises NotImplementedError and
    reading an HDF5-backed file fails with the engine's error."""

    class Encoding:
        HDF5 = 0
        ASCII = 1

    def __init__(self, *args):
        # XDMFFile(filename) or XDMFFile(comm, filename) (comm ignored: serial)
        name = os.fspath(args[-1])
        self.name = name

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        return False

    def close(self):
        pass

    def write(self, obj, encoding=Encoding.ASCII):
        from .cpp import Mesh
        from .function import Function
        if encoding != XDMFFile.Encoding.ASCII:
            raise NotImplementedError("XDMF with HDF5 encoding needs HDF5 (not in this build); "
                                      "use XDMFFile.Encoding.ASCII")
        if isinstance(obj, Mesh):
            call("db2_mesh_write_xdmf", obj.handle, os.fsencode(self.name), None, 0, None)
        elif isinstance(obj, Function):
            V = obj.function_space()
            if V.degree() != 1:
                raise NotImplementedError("XDMF output of P1 (vertex) functions is provided")
            mesh = V.mesh()
            vs = V.value_size()
            if vs > 1 and V.reordered():
                raise NotImplementedError("XDMF output of vector functions on reordered spaces")
            # by vertex: component-major dofs -> (nv, vs)
            vals = np.ascontiguousarray(
                obj.vertex_tensor().detach().cpu().numpy().reshape(vs, -1).T, np.float64)
            name = obj.name if isinstance(obj.name, str) else obj.name()
            call("db2_mesh_write_xdmf", mesh.handle, os.fsencode(self.name),
                 C.c_void_p(vals.ctypes.data), vs, name.encode())
        else:
            raise NotImplementedError(f"XDMFFile.write({type(obj).__name__}) is not provided")

    def read(self, mesh):
        """Read the file's mesh into ``mesh`` (its previous contents are
        released; spaces built on it keep their own reference)."""
        from .cpp import Mesh
        if not isinstance(mesh, Mesh):
            raise NotImplementedError("XDMFFile.read is provided for meshes")
        h = C.c_void_p()
        call("db2_mesh_read_xdmf", os.fsencode(self.name), C.byref(h))
        old = mesh._h
        Mesh.__init__(mesh, _handle=h)
        if old is not None:
            _capi.lib().db2_mesh_destroy(old)
        return mesh
