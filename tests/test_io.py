"""DOLFIN XML input/output of meshes and vectors (host only; no GPU)."""
import ctypes as C
import os

import numpy as np
import pytest

import dolfin_b200 as d2
from dolfin_b200 import _capi

# The reference tetrahedron in DOLFIN's XML mesh format (the layout that
# dolfin/io/XMLMesh.cpp reads; the reference's test_assembler.py uses such a
# file), with the cell's vertices listed out of order on purpose.
TET_XML = """<?xml version="1.0" encoding="UTF-8"?>
<dolfin xmlns:dolfin="http://www.fenics.org/dolfin/">
  <!-- one tetrahedron -->
  <mesh celltype="tetrahedron" dim="3">
    <vertices size="4">
      <vertex index="0" x="0" y="0" z="0" />
      <vertex index="1" x="1" y="0" z="0" />
      <vertex index="2" x="0" y="1" z="0" />
      <vertex index="3" x="0" y="0" z="1" />
    </vertices>
    <cells size="1">
      <tetrahedron index="0" v0="3" v1="0" v2="2" v3="1"/>
    </cells>
  </mesh>
</dolfin>
"""


def test_read_tetrahedron_xml(tmp_path):
    p = tmp_path / "tetrahedron.xml"
    p.write_text(TET_XML)
    m = d2.Mesh(str(p))
    assert m.num_vertices() == 4 and m.num_cells() == 1
    assert m.cells().tolist() == [[0, 1, 2, 3]]  # ordered as MeshEditor::close leaves it
    assert np.array_equal(m.coordinates(), [[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]])


@pytest.mark.parametrize("tdim", [2, 3])
def test_mesh_round_trip_is_exact(tmp_path, tdim):
    from dolfin_b200 import synthetic
    m = d2.UnitSquareMesh(5, 4) if tdim == 2 else d2.UnitCubeMesh(3, 2, 2)
    m.set_coordinates(synthetic.jitter_interior(m.coordinates(), 4, 0.2, 3))
    p = tmp_path / "m.xml"
    d2.File(str(p)) << m
    m2 = d2.Mesh(str(p))
    assert np.array_equal(m2.cells(), m.cells())
    assert np.array_equal(m2.coordinates(), m.coordinates())  # 17 significant digits


def test_vector_round_trip_is_exact(tmp_path):
    x = np.random.default_rng(1).standard_normal(197)
    p = os.fsencode(str(tmp_path / "x.xml"))
    _capi.call("db2_vector_write_xml", p, x.shape[0], C.c_void_p(x.ctypes.data))
    n = C.c_int64(0)
    _capi.call("db2_vector_read_xml", p, C.byref(n), None)
    y = np.empty(n.value)
    _capi.call("db2_vector_read_xml", p, C.byref(n), C.c_void_p(y.ctypes.data))
    assert n.value == 197 and np.array_equal(x, y)


def test_bad_files_raise(tmp_path):
    with pytest.raises(_capi.DB2Error):
        d2.Mesh(str(tmp_path / "missing.xml"))
    p = tmp_path / "hex.xml"
    p.write_text(TET_XML.replace('celltype="tetrahedron"', 'celltype="hexahedron"'))
    with pytest.raises(_capi.DB2Error):
        d2.Mesh(str(p))
    p.write_text(TET_XML.replace('v3="1"', 'v3="7"'))
    with pytest.raises(_capi.DB2Error):
        d2.Mesh(str(p))
    with pytest.raises(NotImplementedError):
        d2.File(str(tmp_path / "m.pvd"))
