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


# A two-triangle mesh in the layout XDMFFile::write(mesh, Encoding::ASCII)
# produces (dolfin/io/XDMFFile.cpp add_mesh / add_topology_data /
# add_geometry_data / add_data_item), vertex lists deliberately unsorted.
TRI_XDMF = """<?xml version="1.0"?>
<!DOCTYPE Xdmf SYSTEM "Xdmf.dtd" []>
<Xdmf Version="3.0" xmlns:xi="http://www.w3.org/2001/XInclude">
  <Domain>
    <Grid Name="mesh" GridType="Uniform">
      <Topology NumberOfElements="2" TopologyType="Triangle" NodesPerElement="3">
        <DataItem Dimensions="2 3" NumberType="UInt" Format="XML">0 1 3
2 3 0</DataItem>
      </Topology>
      <Geometry GeometryType="XY">
        <DataItem Dimensions="4 2" Format="XML">0 0
1 0
1 1
0 1</DataItem>
      </Geometry>
    </Grid>
  </Domain>
</Xdmf>
"""


def test_read_xdmf_ascii_mesh(tmp_path):
    p = tmp_path / "two.xdmf"
    p.write_text(TRI_XDMF)
    m = d2.Mesh(str(p))
    assert m.num_vertices() == 4 and m.num_cells() == 2
    assert m.cells().tolist() == [[0, 1, 3], [0, 2, 3]]  # sorted, as Mesh::order leaves them
    assert np.array_equal(m.coordinates(), [[0, 0], [1, 0], [1, 1], [0, 1]])
    m2 = d2.UnitSquareMesh(1, 1)
    with d2.XDMFFile(str(p)) as f:
        f.read(m2)  # XDMFFile.read(mesh) replaces the mesh's contents
    assert m2.num_cells() == 2 and np.array_equal(m2.cells(), m.cells())


@pytest.mark.parametrize("tdim", [2, 3])
def test_xdmf_mesh_round_trip_is_exact(tmp_path, tdim):
    from dolfin_b200 import synthetic
    m = d2.UnitSquareMesh(5, 4) if tdim == 2 else d2.UnitCubeMesh(3, 2, 2)
    m.set_coordinates(synthetic.jitter_interior(m.coordinates(), 4, 0.2, 3))
    p = tmp_path / "m.xdmf"
    with d2.XDMFFile(str(p)) as f:
        f.write(m)
    text = p.read_text()
    assert ('TopologyType="Tetrahedron"' if tdim == 3 else 'TopologyType="Triangle"') in text
    assert 'Format="XML"' in text and 'NumberType="UInt"' in text
    m2 = d2.Mesh(str(p))
    assert np.array_equal(m2.cells(), m.cells())
    assert np.array_equal(m2.coordinates(), m.coordinates())  # 17 significant digits


def test_xdmf_p1_function_attribute(tmp_path):
    import xml.etree.ElementTree as ET
    m = d2.UnitCubeMesh(2, 2, 2)
    W = d2.FunctionSpace(m, "Lagrange", 1)
    vals = np.arange(m.num_vertices(), dtype=np.float64) * 0.5
    f = d2.Function(W, vals, name="kappa")
    p = tmp_path / "f.xdmf"
    d2.XDMFFile(str(p)).write(f)
    root = ET.parse(p).getroot()
    attr = root.find("./Domain/Grid/Attribute")
    assert attr.get("Name") == "kappa" and attr.get("Center") == "Node"
    assert attr.get("AttributeType") == "Scalar"
    got = np.array(attr.find("DataItem").text.split(), dtype=np.float64)
    assert np.array_equal(got, vals)
    V = d2.VectorFunctionSpace(m, "Lagrange", 1)
    u = d2.Function(V, np.arange(V.dim(), dtype=np.float64), name="u")
    d2.XDMFFile(str(p)).write(u)
    attr = ET.parse(p).getroot().find("./Domain/Grid/Attribute")
    assert attr.get("AttributeType") == "Vector"
    got = np.array(attr.find("DataItem").text.split(), dtype=np.float64).reshape(-1, 3)
    nv = m.num_vertices()
    assert np.array_equal(got, np.arange(3 * nv, dtype=np.float64).reshape(3, nv).T)


def test_xdmf_rejects_hdf5_and_bad_files(tmp_path):
    p = tmp_path / "h5.xdmf"
    p.write_text(TRI_XDMF.replace('NumberType="UInt" Format="XML"', 'NumberType="UInt" Format="HDF"'))
    with pytest.raises(_capi.DB2Error, match="HDF5"):
        d2.Mesh(str(p))
    p.write_text(TRI_XDMF.replace('Dimensions="2 3"', 'Dimensions="3 3"'))
    with pytest.raises(_capi.DB2Error, match="DataItem holds"):
        d2.Mesh(str(p))
    p.write_text(TRI_XDMF.replace("2 3 0</DataItem>", "2 3 7</DataItem>"))
    with pytest.raises(_capi.DB2Error, match="vertex"):
        d2.Mesh(str(p))
    # an index beyond 32 bits is refused, not wrapped to a valid vertex
    p.write_text(TRI_XDMF.replace("2 3 0</DataItem>", "2 3 4294967296</DataItem>"))
    with pytest.raises(_capi.DB2Error, match="bad index"):
        d2.Mesh(str(p))
    # Dimensions larger than the data can hold are refused before reserving
    p.write_text(TRI_XDMF.replace('Dimensions="2 3"', 'Dimensions="1000000000000 3"'))
    with pytest.raises(_capi.DB2Error, match="exceed its data"):
        d2.Mesh(str(p))
    p.write_text(TRI_XDMF.replace('TopologyType="Triangle"', 'TopologyType="Quadrilateral"'))
    with pytest.raises(_capi.DB2Error, match="TopologyType"):
        d2.Mesh(str(p))
    with pytest.raises(NotImplementedError):
        d2.XDMFFile(str(tmp_path / "x.xdmf")).write(d2.UnitSquareMesh(1, 1), encoding=d2.XDMFFile.Encoding.HDF5)
