"""File -- DOLFIN XML input/output of meshes and vectors (dolfin.File with
the .xml suffix: dolfin/io/File.cpp, XMLFile.cpp, XMLMesh.cpp, XMLVector.cpp).

    File("mesh.xml") << mesh        File("b.xml") << b
    mesh = Mesh("mesh.xml")         File("b.xml") >> b

The files are read and written by the engine library (C++); vectors are
copied between device and host around the call.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

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
