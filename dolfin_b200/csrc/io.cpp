// io.cpp -- DOLFIN XML files for meshes and vectors (host only).
//
// Mesh: XMLMesh::read_mesh / XMLMesh::write (dolfin/io/XMLMesh.cpp:88-150,
// :426-500):
//   <dolfin> <mesh celltype="tetrahedron|triangle" dim="g">
//     <vertices size="nv"> <vertex index="i" x=".." y=".." [z=".."]/> ...
//     <cells size="nc"> <tetrahedron index="c" v0=".." v1=".." v2=".." v3=".."/> ...
// Vectors: XMLVector / XMLArray (dolfin/io/XMLVector.cpp:54-140,
// dolfin/io/XMLArray.h:95-125):
//   <dolfin> <vector> <array type="double" size="n"> <element index="i" value=".."/> ...
// The reader is a small tag scanner for exactly these documents (no DTD,
// entities or namespaces beyond the root's attribute).  Cells are stored with
// their vertices sorted ascending, as MeshEditor::close -> Mesh::order leaves
// a freshly read mesh (TetrahedronCell::order, dolfin/mesh/TetrahedronCell.cpp:455).
#include <algorithm>
#include <limits>
#include <cctype>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <type_traits>
#include <vector>

#include "internal.h"

namespace db2 {
namespace {

struct Tag {
  std::string name;
  std::map<std::string, std::string> attr;
  size_t body = 0;  // offset just past the start tag (element text begins)
};

// All element start tags of the document, in order ('<?', '<!' and end tags
// skipped).
std::vector<Tag> scan_tags(const std::string& s) {
  std::vector<Tag> tags;
  size_t i = 0;
  while ((i = s.find('<', i)) != std::string::npos) {
    if (i + 1 < s.size() && (s[i + 1] == '?' || s[i + 1] == '!' || s[i + 1] == '/')) {
      if (s.compare(i, 4, "<!--") == 0) {
        const size_t e = s.find("-->", i);
        i = e == std::string::npos ? s.size() : e + 3;
      } else {
        ++i;
      }
      continue;
    }
    const size_t end = s.find('>', i);
    if (end == std::string::npos) fail(DB2_ERR_ARGUMENT, "XML: unterminated tag");
    Tag t;
    size_t p = i + 1;
    while (p < end && !isspace((unsigned char)s[p]) && s[p] != '/') t.name += s[p++];
    while (p < end) {
      while (p < end && (isspace((unsigned char)s[p]) || s[p] == '/')) ++p;
      if (p >= end) break;
      std::string key;
      while (p < end && s[p] != '=' && !isspace((unsigned char)s[p])) key += s[p++];
      while (p < end && s[p] != '"' && s[p] != '\'') ++p;
      if (p >= end) fail(DB2_ERR_ARGUMENT, "XML: attribute %s without a value", key.c_str());
      const char q = s[p++];
      const size_t ve = s.find(q, p);
      if (ve == std::string::npos || ve > end) fail(DB2_ERR_ARGUMENT, "XML: bad attribute %s", key.c_str());
      t.attr[key] = s.substr(p, ve - p);
      p = ve + 1;
    }
    t.body = end + 1;
    tags.push_back(std::move(t));
    i = end + 1;
  }
  return tags;
}

std::string read_file(const char* path) {
  std::ifstream f(path, std::ios::binary);
  if (!f) fail(DB2_ERR_ARGUMENT, "cannot open %s", path);
  std::ostringstream ss;
  ss << f.rdbuf();
  return ss.str();
}

const std::string& need_attr(const Tag& t, const char* key) {
  auto it = t.attr.find(key);
  if (it == t.attr.end()) fail(DB2_ERR_ARGUMENT, "XML: <%s> lacks attribute %s", t.name.c_str(), key);
  return it->second;
}

int64_t to_int(const std::string& v) {
  char* e = nullptr;
  const long long x = std::strtoll(v.c_str(), &e, 10);
  if (e == v.c_str() || *e) fail(DB2_ERR_ARGUMENT, "XML: '%s' is not an integer", v.c_str());
  return x;
}

double to_double(const std::string& v) {
  char* e = nullptr;
  const double x = std::strtod(v.c_str(), &e);
  if (e == v.c_str()) fail(DB2_ERR_ARGUMENT, "XML: '%s' is not a number", v.c_str());
  return x;
}

void write_file(const char* path, const std::string& s) {
  std::ofstream f(path, std::ios::binary);
  if (!f) fail(DB2_ERR_ARGUMENT, "cannot write %s", path);
  f << s;
  if (!f) fail(DB2_ERR_ARGUMENT, "write to %s failed", path);
}

std::string fmt17(double x) {
  char b[40];
  std::snprintf(b, sizeof(b), "%.17g", x);
  return b;
}

}  // namespace

std::shared_ptr<Mesh> read_mesh_xml(const char* path) {
  const std::vector<Tag> tags = scan_tags(read_file(path));
  const Tag* mesh = nullptr;
  for (const Tag& t : tags)
    if (t.name == "mesh") { mesh = &t; break; }
  if (!mesh) fail(DB2_ERR_ARGUMENT, "%s: no <mesh> element", path);
  const std::string& ct = need_attr(*mesh, "celltype");
  const int tdim = ct == "tetrahedron" ? 3 : (ct == "triangle" ? 2 : 0);
  if (!tdim) fail(DB2_ERR_UNSUPPORTED, "%s: cell type %s (triangle/tetrahedron provided)", path, ct.c_str());
  const int64_t gdim = to_int(need_attr(*mesh, "dim"));
  if (gdim != tdim) fail(DB2_ERR_UNSUPPORTED, "%s: geometric dimension %lld != topological %d", path, (long long)gdim, tdim);
  int64_t nv = -1, nc = -1;
  std::vector<double> x;
  std::vector<uint32_t> cells;
  std::vector<uint8_t> seen_v, seen_c;
  const char* axes[3] = {"x", "y", "z"};
  for (const Tag& t : tags) {
    if (t.name == "vertices") {
      nv = to_int(need_attr(t, "size"));
      x.assign(size_t(nv) * tdim, 0.0);
      seen_v.assign(nv, 0);
    } else if (t.name == "cells") {
      nc = to_int(need_attr(t, "size"));
      cells.assign(size_t(nc) * (tdim + 1), 0);
      seen_c.assign(nc, 0);
    } else if (t.name == "vertex") {
      if (nv < 0) fail(DB2_ERR_ARGUMENT, "%s: <vertex> outside <vertices>", path);
      const int64_t i = to_int(need_attr(t, "index"));
      if (i < 0 || i >= nv || seen_v[i]) fail(DB2_ERR_INDEX, "%s: vertex index %lld", path, (long long)i);
      seen_v[i] = 1;
      for (int r = 0; r < tdim; ++r) x[i * tdim + r] = to_double(need_attr(t, axes[r]));
    } else if (t.name == ct) {
      if (nc < 0) fail(DB2_ERR_ARGUMENT, "%s: <%s> outside <cells>", path, ct.c_str());
      const int64_t c = to_int(need_attr(t, "index"));
      if (c < 0 || c >= nc || seen_c[c]) fail(DB2_ERR_INDEX, "%s: cell index %lld", path, (long long)c);
      seen_c[c] = 1;
      for (int a = 0; a <= tdim; ++a) {
        const std::string key = "v" + std::to_string(a);
        const int64_t v = to_int(need_attr(t, key.c_str()));
        if (v < 0 || v >= nv) fail(DB2_ERR_INDEX, "%s: cell %lld vertex %lld", path, (long long)c, (long long)v);
        cells[c * (tdim + 1) + a] = uint32_t(v);
      }
      std::sort(cells.begin() + c * (tdim + 1), cells.begin() + (c + 1) * (tdim + 1));
    }
  }
  if (nv < 0 || nc < 0) fail(DB2_ERR_ARGUMENT, "%s: missing <vertices> or <cells>", path);
  if (std::count(seen_v.begin(), seen_v.end(), 0) || std::count(seen_c.begin(), seen_c.end(), 0))
    fail(DB2_ERR_ARGUMENT, "%s: fewer vertices/cells than the declared sizes", path);
  return make_mesh(tdim, nv, x.data(), nc, cells.data());
}

void write_mesh_xml(const Mesh& m, const char* path) {
  std::string s = "<?xml version=\"1.0\"?>\n<dolfin xmlns:dolfin=\"http://fenicsproject.org\">\n";
  const char* ct = m.tdim == 3 ? "tetrahedron" : "triangle";
  s += std::string("  <mesh celltype=\"") + ct + "\" dim=\"" + std::to_string(m.tdim) + "\">\n";
  s += "    <vertices size=\"" + std::to_string(m.nv) + "\">\n";
  const char* axes[3] = {"x", "y", "z"};
  for (int64_t v = 0; v < m.nv; ++v) {
    s += "      <vertex index=\"" + std::to_string(v) + "\"";
    for (int r = 0; r < m.tdim; ++r) s += std::string(" ") + axes[r] + "=\"" + fmt17(m.x[v * m.tdim + r]) + "\"";
    s += " />\n";
  }
  s += "    </vertices>\n    <cells size=\"" + std::to_string(m.nc) + "\">\n";
  for (int64_t c = 0; c < m.nc; ++c) {
    s += std::string("      <") + ct + " index=\"" + std::to_string(c) + "\"";
    for (int a = 0; a <= m.tdim; ++a)
      s += " v" + std::to_string(a) + "=\"" + std::to_string(m.cells[c * (m.tdim + 1) + a]) + "\"";
    s += " />\n";
  }
  s += "    </cells>\n  </mesh>\n</dolfin>\n";
  write_file(path, s);
}

void write_vector_xml(const char* path, int64_t n, const double* x) {
  if (n <= 0) fail(DB2_ERR_ARGUMENT, "write vector to XML file: size is zero");
  std::string s = "<?xml version=\"1.0\"?>\n<dolfin xmlns:dolfin=\"http://fenicsproject.org\">\n";
  s += "  <vector>\n    <array type=\"double\" size=\"" + std::to_string(n) + "\">\n";
  for (int64_t i = 0; i < n; ++i)
    s += "      <element index=\"" + std::to_string(i) + "\" value=\"" + fmt17(x[i]) + "\" />\n";
  s += "    </array>\n  </vector>\n</dolfin>\n";
  write_file(path, s);
}

// ---- XDMF (ASCII encoding) ---------------------------------------------------
// XDMFFile::write(mesh, Encoding::ASCII) / XDMFFile::read(mesh)
// (dolfin/io/XDMFFile.cpp:91-131 add_mesh :1140, add_topology_data :1788,
// add_geometry_data :1831, add_data_item :1879, vtk_cell_type_str :3090):
//   <Xdmf Version="3.0"> <Domain> <Grid Name="mesh" GridType="Uniform">
//     <Topology NumberOfElements="nc" TopologyType="Tetrahedron|Triangle"
//               NodesPerElement="d+1">
//       <DataItem Dimensions="nc d+1" NumberType="UInt" Format="XML"> ... </DataItem>
//     <Geometry GeometryType="XYZ|XY">
//       <DataItem Dimensions="nv d" Format="XML"> ... </DataItem>
// HDF5-backed items (Format="HDF") need HDF5, which this build does not
// have; affine (first-order) simplices with gdim == tdim only.
namespace {

// The whitespace-separated numbers of the DataItem that follows tag `k`.
const Tag& data_item_after(const std::vector<Tag>& tags, size_t k, const char* path) {
  for (size_t j = k + 1; j < tags.size(); ++j)
    if (tags[j].name == "DataItem") {
      auto f = tags[j].attr.find("Format");
      const std::string fmt = f == tags[j].attr.end() ? "XML" : f->second;
      if (fmt != "XML")
        fail(DB2_ERR_UNSUPPORTED, "%s: DataItem Format=\"%s\" (HDF5-backed XDMF needs HDF5; write the "
             "file with ASCII encoding)", path, fmt.c_str());
      return tags[j];
    }
  fail(DB2_ERR_ARGUMENT, "%s: <%s> has no DataItem", path, tags[k].name.c_str());
}

std::vector<int64_t> dims_of(const Tag& t, const char* path) {
  std::vector<int64_t> d;
  std::istringstream in(need_attr(t, "Dimensions"));
  int64_t v;
  while (in >> v) d.push_back(v);
  if (d.size() != 2 || d[0] < 0 || d[1] <= 0 || d[1] > 16 || d[0] > (int64_t(1) << 40))
    fail(DB2_ERR_ARGUMENT, "%s: bad DataItem Dimensions", path);
  return d;
}

template <typename T>
std::vector<T> numbers(const std::string& s, const Tag& t, size_t count, const char* path) {
  const size_t end = s.find('<', t.body);
  // every value takes at least one character of the file, so Dimensions
  // beyond that are refused before reserving
  const size_t avail = (end == std::string::npos ? s.size() : end) - t.body;
  if (count > avail + 1)
    fail(DB2_ERR_SHAPE, "%s: DataItem Dimensions (%zu values) exceed its data", path, count);
  std::vector<T> v;
  v.reserve(count);
  const char* p = s.c_str() + t.body;
  const char* stop = s.c_str() + (end == std::string::npos ? s.size() : end);
  while (v.size() < count) {
    while (p < stop && isspace((unsigned char)*p)) ++p;
    if (p >= stop) break;
    char* e = nullptr;
    if constexpr (std::is_floating_point<T>::value) {
      const double x = std::strtod(p, &e);
      if (e == p) fail(DB2_ERR_ARGUMENT, "%s: bad number in DataItem", path);
      v.push_back(T(x));
    } else {
      const long long x = std::strtoll(p, &e, 10);
      if (e == p || x < 0 || (unsigned long long)x > (unsigned long long)std::numeric_limits<T>::max())
        fail(DB2_ERR_ARGUMENT, "%s: bad index in DataItem", path);
      v.push_back(T(x));
    }
    p = e;
  }
  if (v.size() != count) fail(DB2_ERR_SHAPE, "%s: DataItem holds %zu values, Dimensions say %zu", path, v.size(), count);
  return v;
}

}  // namespace

std::shared_ptr<Mesh> read_mesh_xdmf(const char* path) {
  const std::string s = read_file(path);
  const std::vector<Tag> tags = scan_tags(s);
  size_t kt = tags.size(), kg = tags.size();
  for (size_t k = 0; k < tags.size(); ++k) {
    if (tags[k].name == "Topology" && kt == tags.size()) kt = k;
    if (tags[k].name == "Geometry" && kg == tags.size()) kg = k;
  }
  if (kt == tags.size() || kg == tags.size()) fail(DB2_ERR_ARGUMENT, "%s: no <Topology> / <Geometry>", path);
  std::string tt = need_attr(tags[kt], "TopologyType");
  std::transform(tt.begin(), tt.end(), tt.begin(), [](unsigned char c) { return char(std::tolower(c)); });
  const int tdim = tt == "tetrahedron" ? 3 : (tt == "triangle" ? 2 : 0);
  if (!tdim) fail(DB2_ERR_UNSUPPORTED, "%s: TopologyType %s (Triangle/Tetrahedron provided)", path, tt.c_str());
  const std::string gt = need_attr(tags[kg], "GeometryType");
  const int gdim = gt == "XYZ" ? 3 : (gt == "XY" ? 2 : 0);
  if (gdim != tdim) fail(DB2_ERR_UNSUPPORTED, "%s: GeometryType %s with a %d-D cell (gdim == tdim provided)", path, gt.c_str(), tdim);
  const Tag& ti = data_item_after(tags, kt, path);
  const Tag& gi = data_item_after(tags, kg, path);
  const std::vector<int64_t> td = dims_of(ti, path), gd = dims_of(gi, path);
  if (td[1] != tdim + 1 || gd[1] != gdim) fail(DB2_ERR_SHAPE, "%s: DataItem shapes do not match the cell type", path);
  const int64_t nc = td[0], nv = gd[0];
  std::vector<uint32_t> cells = numbers<uint32_t>(s, ti, size_t(nc) * (tdim + 1), path);
  const std::vector<double> x = numbers<double>(s, gi, size_t(nv) * gdim, path);
  for (int64_t c = 0; c < nc; ++c) {
    for (int a = 0; a <= tdim; ++a)
      if (int64_t(cells[c * (tdim + 1) + a]) >= nv)
        fail(DB2_ERR_INDEX, "%s: cell %lld vertex %u", path, (long long)c, cells[c * (tdim + 1) + a]);
    std::sort(cells.begin() + c * (tdim + 1), cells.begin() + (c + 1) * (tdim + 1));
  }
  return make_mesh(tdim, nv, x.data(), nc, cells.data());
}

// With values (nv x value_size, vertex order) a P1 field is added as a
// node-centred Attribute, as XDMFFile::write(const Function&) does for a
// vertex-based function (:311-397).
void write_mesh_xdmf(const Mesh& m, const char* path, const double* values, int value_size,
                     const char* name) {
  if (values && value_size != 1 && value_size != m.tdim)
    fail(DB2_ERR_SHAPE, "XDMF attribute: value size %d (1 or %d provided)", value_size, m.tdim);
  std::string s = "<?xml version=\"1.0\"?>\n<!DOCTYPE Xdmf SYSTEM \"Xdmf.dtd\" []>\n"
                  "<Xdmf Version=\"3.0\" xmlns:xi=\"http://www.w3.org/2001/XInclude\">\n  <Domain>\n"
                  "    <Grid Name=\"mesh\" GridType=\"Uniform\">\n";
  const int nvc = m.tdim + 1;
  s += "      <Topology NumberOfElements=\"" + std::to_string(m.nc) + "\" TopologyType=\"" +
       (m.tdim == 3 ? "Tetrahedron" : "Triangle") + "\" NodesPerElement=\"" + std::to_string(nvc) + "\">\n";
  s += "        <DataItem Dimensions=\"" + std::to_string(m.nc) + " " + std::to_string(nvc) +
       "\" NumberType=\"UInt\" Format=\"XML\">";
  for (int64_t c = 0; c < m.nc; ++c) {
    s += "\n";
    for (int a = 0; a < nvc; ++a) s += (a ? " " : "") + std::to_string(m.cells[c * nvc + a]);
  }
  s += "\n        </DataItem>\n      </Topology>\n";
  s += std::string("      <Geometry GeometryType=\"") + (m.tdim == 3 ? "XYZ" : "XY") + "\">\n";
  s += "        <DataItem Dimensions=\"" + std::to_string(m.nv) + " " + std::to_string(m.tdim) + "\" Format=\"XML\">";
  for (int64_t v = 0; v < m.nv; ++v) {
    s += "\n";
    for (int r = 0; r < m.tdim; ++r) s += (r ? " " : "") + fmt17(m.x[v * m.tdim + r]);
  }
  s += "\n        </DataItem>\n      </Geometry>\n";
  if (values) {
    const int ncomp = value_size == 1 ? 1 : 3;  // XDMF vectors are 3-component
    s += std::string("      <Attribute Name=\"") + (name && *name ? name : "f") + "\" AttributeType=\"" +
         (value_size == 1 ? "Scalar" : "Vector") + "\" Center=\"Node\">\n";
    s += "        <DataItem Dimensions=\"" + std::to_string(m.nv) + " " + std::to_string(ncomp) + "\" Format=\"XML\">";
    for (int64_t v = 0; v < m.nv; ++v) {
      s += "\n";
      for (int c = 0; c < ncomp; ++c)
        s += (c ? " " : "") + fmt17(c < value_size ? values[v * value_size + c] : 0.0);
    }
    s += "\n        </DataItem>\n      </Attribute>\n";
  }
  s += "    </Grid>\n  </Domain>\n</Xdmf>\n";
  write_file(path, s);
}

int64_t read_vector_xml(const char* path, double* x, int64_t cap) {
  const std::vector<Tag> tags = scan_tags(read_file(path));
  int64_t n = -1;
  for (const Tag& t : tags) {
    if (t.name == "array") {
      if (need_attr(t, "type") != "double") fail(DB2_ERR_UNSUPPORTED, "%s: array type is not double", path);
      n = to_int(need_attr(t, "size"));
      if (!x) return n;
      if (n > cap) fail(DB2_ERR_SHAPE, "%s: %lld values, room for %lld", path, (long long)n, (long long)cap);
    } else if (t.name == "element") {
      if (n < 0) fail(DB2_ERR_ARGUMENT, "%s: <element> outside <array>", path);
      const int64_t i = to_int(need_attr(t, "index"));
      if (i < 0 || i >= n) fail(DB2_ERR_INDEX, "%s: element index %lld", path, (long long)i);
      x[i] = to_double(need_attr(t, "value"));
    }
  }
  if (n < 0) fail(DB2_ERR_ARGUMENT, "%s: no <array> element", path);
  return n;
}

}  // namespace db2
