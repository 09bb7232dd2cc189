// host.cpp -- host-side structures of the engine: meshes, entity numbering,
// dofmaps, the sparsity pattern and the row-gather assembly plan.
//
// These reproduce DOLFIN's serial numbering bit for bit (parameters
// "reorder_dofs_serial" = False) so that the device CSR is index-identical
// to EigenMatrix's; the construction itself is this engine's own
// (bucketed, multi-threaded), not a translation of DOLFIN's.

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <numeric>
#include <thread>

#include "internal.h"

namespace db2 {

void fail(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  throw Error{code, buf};
}

int nverts(int tdim) { return tdim + 1; }
int nedges(int tdim) { return tdim == 3 ? 6 : (tdim == 2 ? 3 : 0); }

// Local edges of the UFC reference cells (TetrahedronCell.cpp:119-124,
// TriangleCell.cpp:106-108).
static const int kTetE[6][2] = {{2, 3}, {1, 3}, {1, 2}, {0, 3}, {0, 2}, {0, 1}};
static const int kTriE[3][2] = {{1, 2}, {0, 2}, {0, 1}};
static const int (*etab(int tdim))[2] { return tdim == 3 ? kTetE : kTriE; }

// Run f(begin, end) over [0, n) on up to hardware_concurrency threads.
template <typename F>
static void parallel_for(int64_t n, F&& f, int64_t min_chunk = 4096) {
  int nt = (int)std::max(1u, std::thread::hardware_concurrency());
  nt = (int)std::min<int64_t>(nt, std::max<int64_t>(1, n / min_chunk));
  if (nt <= 1) {
    f((int64_t)0, n);
    return;
  }
  std::vector<std::thread> th;
  const int64_t chunk = (n + nt - 1) / nt;
  for (int t = 0; t < nt; ++t) {
    const int64_t b = t * chunk, e = std::min(n, b + chunk);
    if (b >= e) break;
    th.emplace_back([&f, b, e] { f(b, e); });
  }
  for (auto& t : th) t.join();
}

// ---------------------------------------------------------------------------
// Meshes
// ---------------------------------------------------------------------------
std::shared_ptr<Mesh> make_mesh(int tdim, int64_t nv, const double* x, int64_t nc,
                                const uint32_t* cells) {
  if (tdim != 2 && tdim != 3) fail(DB2_ERR_UNSUPPORTED, "only triangles and tetrahedra are supported (tdim=%d)", tdim);
  if (nv <= 0 || nc <= 0 || !x || !cells) fail(DB2_ERR_ARGUMENT, "empty mesh");
  if (nc >= (int64_t(1) << 28)) fail(DB2_ERR_UNSUPPORTED, "too many cells (%lld)", (long long)nc);
  auto m = std::make_shared<Mesh>();
  m->tdim = tdim;
  m->nv = nv;
  m->nc = nc;
  m->x.assign(x, x + nv * tdim);
  m->cells.assign(cells, cells + nc * (tdim + 1));
  const int n = tdim + 1;
  for (int64_t c = 0; c < nc; ++c) {
    const uint32_t* v = &m->cells[c * n];
    for (int a = 0; a < n; ++a) {
      if (v[a] >= (uint64_t)nv)
        fail(DB2_ERR_INDEX, "cell %lld references vertex %u >= %lld", (long long)c, v[a], (long long)nv);
      if (a > 0 && v[a] <= v[a - 1])
        fail(DB2_ERR_MESH, "Mesh is not ordered according to the UFC numbering convention "
             "(cell %lld vertices not strictly ascending)", (long long)c);
    }
  }
  return m;
}

// BoxMesh::build_tet: vertices in z-y-x order; six tetrahedra per cube sharing
// the diagonal v0-v7; each cell's vertex list sorted (MeshEditor::close
// orders the mesh).
std::shared_ptr<Mesh> make_unit_cube(int nx, int ny, int nz) {
  if (nx < 1 || ny < 1 || nz < 1) fail(DB2_ERR_ARGUMENT, "BoxMesh has non-positive number of vertices in some dimension");
  const int64_t nv = int64_t(nx + 1) * (ny + 1) * (nz + 1);
  const int64_t nc = int64_t(6) * nx * ny * nz;
  std::vector<double> x(nv * 3);
  std::vector<uint32_t> cells(nc * 4);
  const int64_t sx = nx + 1, sxy = int64_t(nx + 1) * (ny + 1);
  parallel_for(nz + 1, [&](int64_t b, int64_t e) {
    for (int64_t iz = b; iz < e; ++iz)
      for (int iy = 0; iy <= ny; ++iy)
        for (int ix = 0; ix <= nx; ++ix) {
          const int64_t v = iz * sxy + iy * sx + ix;
          x[3 * v + 0] = 0.0 + (double(ix)) * (1.0 - 0.0) / double(nx);
          x[3 * v + 1] = 0.0 + (double(iy)) * (1.0 - 0.0) / double(ny);
          x[3 * v + 2] = 0.0 + (double(iz)) * (1.0 - 0.0) / double(nz);
        }
  }, 1);
  parallel_for(nz, [&](int64_t b, int64_t e) {
    for (int64_t iz = b; iz < e; ++iz)
      for (int iy = 0; iy < ny; ++iy)
        for (int ix = 0; ix < nx; ++ix) {
          const uint32_t v0 = uint32_t(iz * sxy + iy * sx + ix);
          const uint32_t v1 = v0 + 1, v2 = v0 + uint32_t(sx), v3 = v1 + uint32_t(sx);
          const uint32_t v4 = v0 + uint32_t(sxy), v5 = v1 + uint32_t(sxy);
          const uint32_t v6 = v2 + uint32_t(sxy), v7 = v3 + uint32_t(sxy);
          // sorted vertex lists of the six Kuhn tetrahedra
          const uint32_t t[6][4] = {{v0, v1, v3, v7}, {v0, v1, v5, v7}, {v0, v4, v5, v7},
                                    {v0, v2, v3, v7}, {v0, v4, v6, v7}, {v0, v2, v6, v7}};
          const int64_t c0 = 6 * ((iz * ny + iy) * int64_t(nx) + ix);
          std::memcpy(&cells[4 * c0], t, sizeof(t));
        }
  }, 1);
  return make_mesh(3, nv, x.data(), nc, cells.data());
}

// RectangleMesh::build_tri on the unit square.
std::shared_ptr<Mesh> make_unit_square(int nx, int ny, int diagonal) {
  if (nx < 1 || ny < 1) fail(DB2_ERR_ARGUMENT, "RectangleMesh has non-positive number of vertices");
  if (diagonal < 0 || diagonal > 3) fail(DB2_ERR_ARGUMENT, "unknown diagonal %d", diagonal);
  const int64_t nv = int64_t(nx + 1) * (ny + 1), nc = int64_t(2) * nx * ny;
  std::vector<double> x(nv * 2);
  std::vector<uint32_t> cells(nc * 3);
  for (int iy = 0; iy <= ny; ++iy)
    for (int ix = 0; ix <= nx; ++ix) {
      const int64_t v = int64_t(iy) * (nx + 1) + ix;
      x[2 * v + 0] = 0.0 + ((double(ix)) * (1.0 - 0.0) / double(nx));
      x[2 * v + 1] = 0.0 + ((double(iy)) * (1.0 - 0.0) / double(ny));
    }
  int64_t c = 0;
  for (int iy = 0; iy < ny; ++iy) {
    bool left = diagonal == 2 ? !(iy % 2) : diagonal == 3 ? (iy % 2) : diagonal == 1;
    for (int ix = 0; ix < nx; ++ix) {
      const uint32_t v0 = uint32_t(iy * (nx + 1) + ix), v1 = v0 + 1;
      const uint32_t v2 = v0 + uint32_t(nx + 1), v3 = v1 + uint32_t(nx + 1);
      const uint32_t a[3] = {v0, v1, left ? v2 : v3};
      const uint32_t b[3] = {left ? v1 : v0, v2, v3};
      std::memcpy(&cells[3 * c], a, sizeof(a));
      std::memcpy(&cells[3 * (c + 1)], b, sizeof(b));
      c += 2;
      if (diagonal >= 2) left = !left;
    }
  }
  return make_mesh(2, nv, x.data(), nc, cells.data());
}

// Exterior facets: facets (vertex key = the cell's vertices other than local
// vertex f, sorted) that occur in exactly one cell (Facet::exterior()),
// listed in key order -- the facet numbering of
// TopologyComputation::compute_entities_by_key_matching
// (dolfin/mesh/TopologyComputation.cpp:152-330) restricted to the boundary.
// Bucketed by the smallest key vertex, sorted by the rest within a bucket.
void Mesh::compute_exterior_facets() {
  if (have_facets) return;
  const int nvc = nverts(tdim), nf = nvc;
  const int64_t nslots = nc * nf;
  if (nc >= (int64_t(1) << 30)) fail(DB2_ERR_UNSUPPORTED, "too many cells for facet records");
  std::vector<uint32_t> start(nv + 1, 0);
  auto key_of = [&](int64_t c, int f, uint32_t k[3]) {
    int m = 0;
    for (int a = 0; a < nvc; ++a)
      if (a != f) k[m++] = cells[c * nvc + a];  // cell vertices are sorted
    if (m < 3) k[2] = 0;
  };
  for (int64_t c = 0; c < nc; ++c)
    for (int f = 0; f < nf; ++f) {
      uint32_t k[3];
      key_of(c, f, k);
      start[k[0] + 1]++;
    }
  for (int64_t v = 0; v < nv; ++v) start[v + 1] += start[v];
  struct Entry { uint64_t rest; uint32_t slot; };
  std::vector<Entry> bucket(nslots);
  std::vector<uint32_t> fillp(start.begin(), start.end() - 1);
  for (int64_t c = 0; c < nc; ++c)
    for (int f = 0; f < nf; ++f) {
      uint32_t k[3];
      key_of(c, f, k);
      const uint64_t rest = tdim == 3 ? (uint64_t(k[1]) << 32) | k[2] : uint64_t(k[1]);
      bucket[fillp[k[0]]++] = Entry{rest, uint32_t(c << 2 | f)};
    }
  std::vector<uint32_t> count(nv + 1, 0);
  parallel_for(nv, [&](int64_t b, int64_t e) {
    for (int64_t v = b; v < e; ++v) {
      Entry* lo = bucket.data() + start[v];
      Entry* hi = bucket.data() + start[v + 1];
      std::sort(lo, hi, [](const Entry& x, const Entry& y) {
        return x.rest < y.rest || (x.rest == y.rest && x.slot < y.slot);
      });
      uint32_t u = 0;
      for (Entry* it = lo; it != hi;) {
        Entry* j = it + 1;
        while (j != hi && j->rest == it->rest) ++j;
        if (j - it == 1) ++u;
        it = j;
      }
      count[v + 1] = u;
    }
  });
  for (int64_t v = 0; v < nv; ++v) count[v + 1] += count[v];
  ext_facets.assign(count[nv], 0);
  parallel_for(nv, [&](int64_t b, int64_t e) {
    for (int64_t v = b; v < e; ++v) {
      uint32_t o = count[v];
      Entry* lo = bucket.data() + start[v];
      Entry* hi = bucket.data() + start[v + 1];
      for (Entry* it = lo; it != hi;) {
        Entry* j = it + 1;
        while (j != hi && j->rest == it->rest) ++j;
        if (j - it == 1) ext_facets[o++] = it->slot;
        it = j;
      }
    }
  });
  have_facets = true;
}

// Exterior-facet plan (see FacetPlan).  Facet nodes in canonical facet order:
// the facet's vertices (ascending local index), then for P2 its edges in the
// local edge order of a triangle ((1,2), (0,2), (0,1)) or the one edge of an
// interval, in facet-local vertex indices.
void build_facet_plan(Pattern& P) {
  if (P.facets) return;
  const Space& V = *P.V;
  Mesh& m = *V.mesh;
  m.compute_exterior_facets();
  const int D = m.tdim, nvc = nverts(D), k = V.k;
  const int nfe = V.degree == 2 ? (D == 3 ? 3 : 1) : 0;
  const int kf = D + nfe;
  static const int kFE3[3][2] = {{1, 2}, {0, 2}, {0, 1}};
  static const int kFE2[1][2] = {{0, 1}};
  const int (*FE)[2] = D == 3 ? kFE3 : kFE2;
  const int (*CE)[2] = etab(D);
  auto cell_edge = [&](int a, int b) {
    for (int e = 0; e < nedges(D); ++e)
      if ((CE[e][0] == a && CE[e][1] == b) || (CE[e][0] == b && CE[e][1] == a)) return e;
    return -1;
  };
  auto facet_edge = [&](int p, int q) {
    for (int e = 0; e < nfe; ++e)
      if ((FE[e][0] == p && FE[e][1] == q) || (FE[e][0] == q && FE[e][1] == p)) return e;
    return -1;
  };
  const int64_t nfac = int64_t(m.ext_facets.size());
  // facet nodes (global) and facet vertex ids of every exterior facet
  std::vector<uint32_t> fnode(size_t(nfac) * kf), fvert(size_t(nfac) * D);
  for (int64_t i = 0; i < nfac; ++i) {
    const uint32_t c = m.ext_facets[i] >> 2, fl = m.ext_facets[i] & 3u;
    int av[3], mm = 0;
    for (int a = 0; a < nvc; ++a)
      if (a != int(fl)) av[mm++] = a;
    for (int t = 0; t < D; ++t) {
      fnode[i * kf + t] = V.cell_nodes[int64_t(c) * k + av[t]];
      fvert[i * D + t] = m.cells[int64_t(c) * nvc + av[t]];
    }
    for (int e = 0; e < nfe; ++e)
      fnode[i * kf + D + e] = V.cell_nodes[int64_t(c) * k + nvc + cell_edge(av[FE[e][0]], av[FE[e][1]])];
  }
  auto F = std::make_unique<FacetPlan>();
  F->kf = kf;
  // incidences grouped by node, in facet order within a node
  std::vector<uint32_t> cnt(V.nnodes + 1, 0);
  for (uint32_t n : fnode) cnt[n + 1]++;
  for (int64_t n = 0; n < V.nnodes; ++n) cnt[n + 1] += cnt[n];
  std::vector<uint32_t> order(fnode.size());
  {
    std::vector<uint32_t> fill(cnt.begin(), cnt.end() - 1);
    for (size_t s = 0; s < fnode.size(); ++s) order[fill[fnode[s]]++] = uint32_t(s);
  }
  F->binc_ptr.push_back(0);
  for (int64_t n = 0; n < V.nnodes; ++n)
    if (cnt[n + 1] > cnt[n]) {
      F->bnode.push_back(uint32_t(n));
      F->binc_ptr.push_back(cnt[n + 1]);
    }
  const size_t ninc = order.size();
  F->bverts.resize(ninc * D);
  F->bslot.assign(ninc * 8, 0);
  for (size_t s = 0; s < ninc; ++s) {
    const uint32_t e = order[s];
    const int64_t i = e / kf;
    const int t = int(e % kf);
    const uint32_t node = fnode[e];
    // relabelled facet vertex order: row vertex first, or row edge's two ends
    int ord[3], mm = 0;
    bool used[3] = {false, false, false};
    auto put = [&](int a) {
      ord[mm++] = a;
      used[a] = true;
    };
    if (t < D) {
      put(t);
    } else {
      put(FE[t - D][0]);
      put(FE[t - D][1]);
    }
    for (int a = 0; a < D; ++a)
      if (!used[a]) put(a);
    for (int a = 0; a < D; ++a) F->bverts[s * D + a] = fvert[i * D + ord[a]];
    // column slots of the relabelled facet nodes within the row of `node`
    const int32_t* rb = P.node_cols.data() + P.node_rowptr[node];
    const int32_t* re = P.node_cols.data() + P.node_rowptr[node + 1];
    for (int j = 0; j < kf; ++j) {
      int src = j < D ? ord[j] : D + facet_edge(ord[FE[j - D][0]], ord[FE[j - D][1]]);
      const uint32_t col = fnode[i * kf + src];
      const int32_t* it = std::lower_bound(rb, re, int32_t(col));
      if (it == re || *it != int32_t(col)) fail(DB2_ERR_INDEX, "facet node missing from the pattern");
      F->bslot[s * 8 + j] = uint8_t(it - rb);
    }
  }
  P.facets = std::move(F);
}

const FacetPlan& Pattern::facet_plan() {
  if (!facets || !facets->d_binc_ptr.ptr) {
    build_facet_plan(*this);
    FacetPlan& F = *facets;
    auto up = [](DeviceBuffer& d, const auto& v) {
      if (!v.empty()) d.upload(v.data(), v.size() * sizeof(v[0]));
    };
    up(F.d_bnode, F.bnode);
    up(F.d_binc_ptr, F.binc_ptr);
    up(F.d_bverts, F.bverts);
    up(F.d_bslot, F.bslot);
  }
  return *facets;
}

// Entity numbering of edges: equivalent to sorting all (cell, local edge)
// entries by their sorted vertex key and numbering distinct keys in order
// (TopologyComputation::compute_entities_by_key_matching,
// dolfin/mesh/TopologyComputation.cpp:152-330).  Done as a bucket sort on the
// smaller vertex, then a small sort of the larger vertex within each bucket.
void Mesh::compute_edges() {
  if (have_edges) return;
  const int ne_c = nedges(tdim), nvc = nverts(tdim);
  const int (*E)[2] = etab(tdim);
  std::vector<uint32_t> start(nv + 1, 0);
  for (int64_t c = 0; c < nc; ++c)
    for (int e = 0; e < ne_c; ++e) {
      const uint32_t p = cells[c * nvc + E[e][0]];  // cell vertices are sorted: p < q
      start[p + 1]++;
    }
  for (int64_t v = 0; v < nv; ++v) start[v + 1] += start[v];
  const int64_t nslots = nc * ne_c;
  if (nslots >= (int64_t(1) << 32)) fail(DB2_ERR_UNSUPPORTED, "too many cell edges");
  std::vector<uint64_t> bucket(nslots);  // (q << 32) | slot... slot needs 32 bits
  std::vector<uint32_t> fillp(start.begin(), start.end() - 1);
  for (int64_t c = 0; c < nc; ++c)
    for (int e = 0; e < ne_c; ++e) {
      const uint32_t p = cells[c * nvc + E[e][0]], q = cells[c * nvc + E[e][1]];
      bucket[fillp[p]++] = (uint64_t(q) << 32) | uint32_t(c * ne_c + e);
    }
  std::vector<uint32_t> nuniq(nv + 1, 0);
  parallel_for(nv, [&](int64_t b, int64_t e) {
    for (int64_t v = b; v < e; ++v) {
      auto* lo = bucket.data() + start[v];
      auto* hi = bucket.data() + start[v + 1];
      std::sort(lo, hi);
      uint32_t u = 0;
      uint64_t prev = ~uint64_t(0);
      for (auto* it = lo; it != hi; ++it) {
        const uint64_t q = *it >> 32;
        if (q != prev) { ++u; prev = q; }
      }
      nuniq[v + 1] = u;
    }
  });
  for (int64_t v = 0; v < nv; ++v) nuniq[v + 1] += nuniq[v];
  ne = nuniq[nv];
  cell_edges.assign(nslots, 0);
  edge_vertices.assign(size_t(ne) * 2, 0);
  parallel_for(nv, [&](int64_t b, int64_t e) {
    for (int64_t v = b; v < e; ++v) {
      int64_t id = int64_t(nuniq[v]) - 1;
      uint64_t prev = ~uint64_t(0);
      for (uint32_t s = start[v]; s < start[v + 1]; ++s) {
        const uint64_t q = bucket[s] >> 32;
        if (q != prev) {
          ++id;
          prev = q;
          edge_vertices[2 * id] = uint32_t(v);
          edge_vertices[2 * id + 1] = uint32_t(q);
        }
        cell_edges[bucket[s] & 0xffffffffu] = uint32_t(id);
      }
    }
  });
  have_edges = true;
}

// ---------------------------------------------------------------------------
// Function spaces: natural UFC numbering (DofMapBuilder.cpp:253-272):
// vertex dofs = vertex index; P2 edge dofs = nv + edge index at local slots
// nv_cell.. in local-edge order; vector spaces component-major.
// ---------------------------------------------------------------------------
std::shared_ptr<Space> make_space(std::shared_ptr<Mesh> m, int degree, int vsize) {
  if (degree != 1 && degree != 2) fail(DB2_ERR_UNSUPPORTED, "Lagrange degree %d not provided (1 or 2)", degree);
  if (vsize != 1 && vsize != m->tdim) fail(DB2_ERR_UNSUPPORTED, "value size %d not provided (1 or %d)", vsize, m->tdim);
  auto V = std::make_shared<Space>();
  V->mesh = m;
  V->degree = degree;
  V->vsize = vsize;
  const int nvc = nverts(m->tdim), nec = nedges(m->tdim);
  V->k = degree == 1 ? nvc : nvc + nec;
  if (degree == 2) m->compute_edges();
  V->nnodes = m->nv + (degree == 2 ? m->ne : 0);
  if (V->nnodes * vsize >= (int64_t(1) << 31)) fail(DB2_ERR_UNSUPPORTED, "global dimension exceeds int32 (Eigen StorageIndex)");
  V->cell_nodes.resize(m->nc * V->k);
  parallel_for(m->nc, [&](int64_t b, int64_t e) {
    for (int64_t c = b; c < e; ++c) {
      uint32_t* out = &V->cell_nodes[c * V->k];
      for (int a = 0; a < nvc; ++a) out[a] = m->cells[c * nvc + a];
      if (degree == 2)
        for (int j = 0; j < nec; ++j) out[nvc + j] = uint32_t(m->nv + m->cell_edges[c * nec + j]);
    }
  });
  return V;
}

void canonical_perm(int tdim, int li, int perm[4]) {
  const int nvc = nverts(tdim);
  int first[2], nf;
  if (li < nvc) {
    first[0] = li;
    nf = 1;
  } else {
    first[0] = etab(tdim)[li - nvc][0];
    first[1] = etab(tdim)[li - nvc][1];
    nf = 2;
  }
  int n = 0;
  for (int i = 0; i < nf; ++i) perm[n++] = first[i];
  for (int a = 0; a < nvc; ++a)
    if (a != first[0] && (nf == 1 || a != first[1])) perm[n++] = a;
}

void canonical_node_map(int tdim, int degree, int li, int* map) {
  int perm[4];
  canonical_perm(tdim, li, perm);
  const int nvc = nverts(tdim), nec = nedges(tdim);
  for (int a = 0; a < nvc; ++a) map[a] = perm[a];
  if (degree < 2) return;
  const int (*E)[2] = etab(tdim);
  for (int e2 = 0; e2 < nec; ++e2) {
    const int p = perm[E[e2][0]], q = perm[E[e2][1]];
    int found = -1;
    for (int e = 0; e < nec; ++e)
      if ((E[e][0] == p && E[e][1] == q) || (E[e][0] == q && E[e][1] == p)) found = e;
    map[nvc + e2] = nvc + found;
  }
}

// ---------------------------------------------------------------------------
// Sparsity pattern + row-gather plan.
//
// DOLFIN inserts, cell by cell, every (row dof, column dof) pair of the cell
// into per-row dolfin::Set's and sorts the rows (SparsityPatternBuilder::build,
// SparsityPattern::diagonal_pattern(sorted)).  The union is the same as: row
// node i's columns = sorted unique nodes of the cells incident to i.  We
// build it from the node -> (cell, local node) incidence lists, which are
// also the engine's assembly plan: a device thread owning row i visits the
// incident cells in ascending order -- the order in which DOLFIN's cell loop
// adds their contributions to row i.
// ---------------------------------------------------------------------------
// Tiles: contiguous node ranges with at most one row unit (node x trial
// block) per thread whose row segment (one test component) fits
// seg_cap_doubles.

std::vector<Tile> cut_tiles(const Pattern& P, int tile_threads, int seg_cap_doubles, int* max_seg_out,
                            int64_t node_begin, int64_t node_end) {
  const int bs = P.bs;
  const int64_t nn = node_end < 0 ? P.V->nnodes : node_end;
  // P2: vertex nodes [0, nv) precede edge nodes; no tile spans both, so the
  // kernel knows each tile's row kind up front
  const int64_t split = P.V->degree == 2 ? P.V->mesh->nv : -1;
  int max_seg = 0;
  std::vector<Tile> comp0;
  int64_t n0 = node_begin;
  while (n0 < nn) {
    int64_t n1 = n0;
    while (n1 < nn) {
      if (n1 == split && n1 > n0) break;
      const int64_t units = (n1 + 1 - n0) * bs;
      const int64_t seg = int64_t(bs) * (P.node_rowptr[n1 + 1] - P.node_rowptr[n0]);
      if (units > tile_threads || seg > seg_cap_doubles) break;
      ++n1;
    }
    if (n1 == n0) fail(DB2_ERR_UNSUPPORTED, "row of node %lld does not fit one tile", (long long)n0);
    max_seg = std::max<int>(max_seg, int(int64_t(bs) * (P.node_rowptr[n1] - P.node_rowptr[n0])));
    comp0.push_back(Tile{0, int32_t(n0), int32_t(n1), 0});
    n0 = n1;
  }
  std::vector<Tile> all;
  for (int c = 0; c < bs; ++c)
    for (auto t : comp0) {
      t.comp = c;
      all.push_back(t);
    }
  if (max_seg_out) *max_seg_out = max_seg;
  return all;
}

static void build_tiles(Pattern& P, int tile_threads, int seg_cap_doubles) {
  const int bs = P.bs;
  P.tile_threads = tile_threads;
  P.seg_cap_bytes = seg_cap_doubles * 8;
  int max_seg = 0;
  std::vector<Tile> all = cut_tiles(P, tile_threads, seg_cap_doubles, &max_seg, P.row_begin, P.row_end);
  P.seg_cap = max_seg;
  // Group tiles by the shared memory their row segment needs, so that small
  // (e.g. edge-node) tiles are not launched with the largest tile's
  // allocation: one launch per class.
  static const int kClass[] = {4096, 8192, 12288, 16384, 24576, 32768, 49152, 65536,
                               98304, 131072, 163840, 196608, 227 * 1024};
  const int ncls = int(sizeof(kClass) / sizeof(kClass[0]));
  auto cls_of = [&](const Tile& t) {
    const int64_t need = int64_t(bs) * (P.node_rowptr[t.n1] - P.node_rowptr[t.n0]) * 8;
    int k = 0;
    while (k < ncls - 1 && kClass[k] < need) ++k;
    return k;
  };
  std::stable_sort(all.begin(), all.end(), [&](const Tile& a, const Tile& b) { return cls_of(a) < cls_of(b); });
  P.tiles = all;
  P.class_begin.clear();
  P.class_smem.clear();
  for (size_t i = 0; i < all.size(); ++i) {
    const int k = cls_of(all[i]);
    if (i == 0 || k != cls_of(all[i - 1])) {
      P.class_begin.push_back(int32_t(i));
      P.class_smem.push_back(kClass[k]);
    }
  }
  P.class_begin.push_back(int32_t(all.size()));
}

void retile(Pattern& P, int tile_threads, int seg_cap_bytes) {
  if (tile_threads <= 0 || tile_threads > 256 || tile_threads % 32)
    fail(DB2_ERR_ARGUMENT, "tile_threads must be a positive multiple of 32 (<= 256)");
  if (seg_cap_bytes < 1024 || seg_cap_bytes > 220 * 1024)
    fail(DB2_ERR_ARGUMENT, "seg_cap_bytes out of range");
  build_tiles(P, tile_threads, seg_cap_bytes / 8);
  if (P.on_device) P.d_tiles.upload(P.tiles.data(), P.tiles.size() * sizeof(Tile));
}

// Row-partitioned assembly: a rank assembles the node rows [node_begin,
// node_end) completely from the cells around them (their incidence lists),
// with no exchange -- the row-owner analogue of DOLFIN's owned-row ranges
// (SparsityPattern.cpp:200-255).  Only the tile kernel is restricted.
void set_row_range(Pattern& P, int64_t node_begin, int64_t node_end, bool block_storage) {
  const int64_t nn = P.V->nnodes;
  if (node_begin < 0 || node_end < node_begin || node_end > nn)
    fail(DB2_ERR_ARGUMENT, "row range [%lld, %lld) outside [0, %lld)", (long long)node_begin,
         (long long)node_end, (long long)nn);
  if (P.V->reordered() && !(node_begin == 0 && node_end == nn))
    fail(DB2_ERR_UNSUPPORTED, "row ranges are provided for the natural numbering");
  P.row_begin = node_begin;
  P.row_end = node_end == nn ? -1 : node_end;
  P.block_storage = block_storage;
  build_tiles(P, P.tile_threads, P.seg_cap_bytes / 8);
  if (P.on_device) P.d_tiles.upload(P.tiles.data(), P.tiles.size() * sizeof(Tile));
}

OutputLayout output_layout(const Pattern& P) {
  const int64_t bs = P.bs;
  if (!P.block_storage) return OutputLayout{bs * P.nnz_node, 0, P.V->nnodes, 0};
  const int64_t n0 = P.row_begin, n1 = P.row_end < 0 ? P.V->nnodes : P.row_end;
  return OutputLayout{bs * (P.node_rowptr[n1] - P.node_rowptr[n0]), bs * P.node_rowptr[n0], n1 - n0, n0};
}

void row_block_size(const Pattern& P, int64_t* nrows, int64_t* nnz) {
  const int64_t n0 = P.row_begin, n1 = P.row_end < 0 ? P.V->nnodes : P.row_end;
  if (nrows) *nrows = (n1 - n0) * P.bs;
  if (nnz) *nnz = int64_t(P.bs) * P.bs * (P.node_rowptr[n1] - P.node_rowptr[n0]);
}

std::shared_ptr<Pattern> make_pattern(std::shared_ptr<Space> V, bool keep_diagonal,
                                      int tile_threads, int seg_cap_bytes) {
  auto P = std::make_shared<Pattern>();
  P->V = V;
  P->keep_diagonal = keep_diagonal;
  P->bs = V->vsize;
  const Mesh& m = *V->mesh;
  const int k = V->k;
  const int64_t nn = V->nnodes, nc = m.nc;
  if (nc * k >= (int64_t(1) << 32)) fail(DB2_ERR_UNSUPPORTED, "too many incidences");

  // node -> incidences, in ascending cell order
  P->inc_ptr.assign(nn + 1, 0);
  for (int64_t i = 0; i < nc * k; ++i) P->inc_ptr[V->cell_nodes[i] + 1]++;
  for (int64_t i = 0; i < nn; ++i) P->inc_ptr[i + 1] += P->inc_ptr[i];
  P->inc.resize(nc * k);
  P->cell_inc.resize(nc * k);
  {
    std::vector<uint32_t> fill(P->inc_ptr.begin(), P->inc_ptr.end() - 1);
    for (int64_t c = 0; c < nc; ++c)
      for (int li = 0; li < k; ++li) {
        const uint32_t node = V->cell_nodes[c * k + li];
        const uint32_t slot = fill[node]++;
        P->inc[slot] = uint32_t(c) | (uint32_t(li) << 28);
        P->cell_inc[c * k + li] = slot;
      }
  }

  // node-level CSR (sorted unique neighbours through cells)
  P->node_rowptr.assign(nn + 1, 0);
  auto neighbours = [&](int64_t i, std::vector<uint32_t>& buf) {
    buf.clear();
    for (uint32_t s = P->inc_ptr[i]; s < P->inc_ptr[i + 1]; ++s) {
      const uint32_t c = P->inc[s] & 0x0fffffffu;
      buf.insert(buf.end(), &V->cell_nodes[int64_t(c) * k], &V->cell_nodes[int64_t(c) * k] + k);
    }
    std::sort(buf.begin(), buf.end());
    buf.erase(std::unique(buf.begin(), buf.end()), buf.end());
  };
  std::atomic<int64_t> too_long{-1};
  parallel_for(nn, [&](int64_t b, int64_t e) {
    std::vector<uint32_t> buf;
    for (int64_t i = b; i < e; ++i) {
      neighbours(i, buf);
      if (buf.size() > 255) too_long = i;
      P->node_rowptr[i + 1] = int32_t(buf.size());
    }
  });
  if (too_long >= 0) fail(DB2_ERR_UNSUPPORTED, "node %lld has more than 255 neighbours", (long long)too_long.load());
  int64_t acc = 0;
  for (int64_t i = 0; i < nn; ++i) {
    acc += P->node_rowptr[i + 1];
    if (acc * P->bs * P->bs >= (int64_t(1) << 31)) fail(DB2_ERR_UNSUPPORTED, "nnz exceeds int32 (Eigen StorageIndex)");
    P->node_rowptr[i + 1] = int32_t(acc);
  }
  P->nnz_node = acc;
  P->nnz = acc * P->bs * P->bs;
  P->nrows = nn * P->bs;
  P->node_cols.resize(acc);

  // column slots of each incidence's (relabelled) cell nodes
  P->kp = (k + 3) / 4 * 4;
  P->pos.assign(P->inc.size() * P->kp, 0);
  std::vector<std::vector<int>> maps(k, std::vector<int>(k));
  for (int li = 0; li < k; ++li) canonical_node_map(m.tdim, V->degree, li, maps[li].data());
  parallel_for(nn, [&](int64_t b, int64_t e) {
    std::vector<uint32_t> buf;
    for (int64_t i = b; i < e; ++i) {
      neighbours(i, buf);
      std::copy(buf.begin(), buf.end(), P->node_cols.begin() + P->node_rowptr[i]);
      for (uint32_t s = P->inc_ptr[i]; s < P->inc_ptr[i + 1]; ++s) {
        const uint32_t c = P->inc[s] & 0x0fffffffu, li = P->inc[s] >> 28;
        const uint32_t* cn = &V->cell_nodes[int64_t(c) * k];
        for (int j = 0; j < k; ++j) {
          const uint32_t node = cn[maps[li][j]];
          P->pos[int64_t(s) * P->kp + j] = uint8_t(std::lower_bound(buf.begin(), buf.end(), node) - buf.begin());
        }
      }
    }
  });

  // 32 row units and 16 KB of row segment per tile: with the classes running
  // concurrently, small tiles pack the SMs best.  Measured on B200 (ms per
  // A+b step, against 64 / 32 KB): P2 tets n=96 1.234 / 1.252, P1 tets n=96
  // 0.228 / 0.232, vector P2 elasticity n=48 1.284 / 1.283.
  if (tile_threads <= 0) tile_threads = 32;
  if (seg_cap_bytes <= 0) seg_cap_bytes = 16 * 1024;
  build_tiles(*P, tile_threads, seg_cap_bytes / 8);
  return P;
}

void Mesh::ensure_device() {
  if (on_device) return;
  upload_coordinates();
  d_cells.upload(cells.data(), cells.size() * sizeof(uint32_t));
  on_device = true;
}

void Space::ensure_device() {
  mesh->ensure_device();
  if (on_device) return;
  d_cell_nodes.upload(cell_nodes.data(), cell_nodes.size() * sizeof(uint32_t));
  if (degree == 2)
    d_edge_vertices.upload(mesh->edge_vertices.data(), mesh->edge_vertices.size() * sizeof(uint32_t));
  on_device = true;
}

void Pattern::ensure_device() {
  V->ensure_device();
  if (on_device) return;
  d_node_rowptr.upload(node_rowptr.data(), node_rowptr.size() * sizeof(int32_t));
  d_inc_ptr.upload(inc_ptr.data(), inc_ptr.size() * sizeof(uint32_t));
  d_inc.upload(inc.data(), inc.size() * sizeof(uint32_t));
  {
    const Mesh& m = *V->mesh;
    const int D = m.tdim, K = V->k, nd = D;
    rs = 2 * nd + K <= 8 ? 8 : 16;
    const int64_t nn = V->nnodes, ngrp = (nn + 31) / 32;
    rec_goff.assign(ngrp + 1, 0);
    for (int64_t g = 0; g < ngrp; ++g) {
      uint32_t mx = 0;
      for (int64_t i = 32 * g; i < std::min(nn, 32 * g + 32); ++i) mx = std::max(mx, inc_ptr[i + 1] - inc_ptr[i]);
      if (uint64_t(rec_goff[g]) + 32ull * mx >= (1ull << 32)) fail(DB2_ERR_UNSUPPORTED, "too many incidence records");
      rec_goff[g + 1] = rec_goff[g] + 32 * mx;
    }
    std::vector<uint8_t> rec(size_t(rec_goff[ngrp]) * rs, 0);
    std::vector<uint8_t> first(size_t(nn) * rs, 0);
    std::atomic<int64_t> escapes{0};
    parallel_for(nn, [&](int64_t b, int64_t e) {
      for (int64_t i = b; i < e; ++i) {
        // edge-node rows: which of the record's slots this incidence is the
        // first to touch (in incidence order), in the record's otherwise
        // unused last offset field -- the kernel stores there instead of adding
        uint64_t seen[4] = {0, 0, 0, 0};
        for (uint32_t s = inc_ptr[i]; s < inc_ptr[i + 1]; ++s) {
          const uint32_t c = inc[s] & 0x0fffffffu, li = inc[s] >> 28;
          int perm[4];
          canonical_perm(D, int(li), perm);
          const uint32_t* cv = &m.cells[size_t(c) * (D + 1)];
          const int nfix = int(li) <= D ? 1 : 2;
          const int64_t base = cv[perm[0]];
          uint8_t* r = &rec[(size_t(rec_goff[i >> 5]) + (i & 31) + 32ull * (s - inc_ptr[i])) * rs];
          for (int a = nfix; a <= D; ++a) {
            const int64_t d = int64_t(cv[perm[a]]) - base;
            // -32768 marks an offset that does not fit: the kernel then
            // reads this incidence's vertices through its cell
            const bool fits = d >= -32767 && d <= 32767;
            if (!fits) escapes.fetch_add(1, std::memory_order_relaxed);
            const int16_t d16 = fits ? int16_t(d) : int16_t(-32768);
            std::memcpy(r + 2 * (a - nfix), &d16, 2);
          }
          std::memcpy(r + 2 * nd, &pos[size_t(s) * kp], size_t(K));
          if (nfix == 2) {
            uint16_t fm = 0;
            for (int j = 0; j < K; ++j) {
              const uint8_t sl = pos[size_t(s) * kp + j];
              if (!(seen[sl >> 6] >> (sl & 63) & 1u)) {
                fm = uint16_t(fm | (1u << j));
                seen[sl >> 6] |= uint64_t(1) << (sl & 63);
              }
            }
            std::memcpy(r + 2 * (D - 1), &fm, 2);
          }
          if (s == inc_ptr[i]) std::memcpy(&first[size_t(i) * rs], r, size_t(rs));
        }
      }
    });
    rec_escapes = escapes.load();
    d_rec.upload(rec.data(), rec.size());
    d_rec_goff.upload(rec_goff.data(), rec_goff.size() * sizeof(uint32_t));
    d_rec_first.upload(first.data(), first.size());
  }
  d_cell_inc.upload(cell_inc.data(), cell_inc.size() * sizeof(uint32_t));
  d_tiles.upload(tiles.data(), tiles.size() * sizeof(Tile));
  launch_expand_csr(*this);
  noalloc_prepare_device();
  on_device = true;
}

void Pattern::csr_host(int32_t* rowptr, int32_t* cols) {
  if (!V->reordered()) {
    csr_host_natural(rowptr, cols);
    return;
  }
  if (!reordered.built) build_reordered_csr(*this);
  if (rowptr) std::copy(reordered.rowptr.begin(), reordered.rowptr.end(), rowptr);
  if (cols) std::copy(reordered.cols.begin(), reordered.cols.end(), cols);
}

void Pattern::csr_host_natural(int32_t* rowptr, int32_t* cols) const {
  const int64_t nn = V->nnodes;
  for (int c = 0; c < bs; ++c)
    for (int64_t i = 0; i < nn; ++i) {
      const int64_t r = c * nn + i;
      const int32_t a = node_rowptr[i], L = node_rowptr[i + 1] - a;
      const int64_t rp = int64_t(c) * bs * nnz_node + int64_t(bs) * a;
      if (rowptr) rowptr[r] = int32_t(rp);
      if (cols)
        for (int e = 0; e < bs; ++e)
          for (int t = 0; t < L; ++t) cols[rp + int64_t(e) * L + t] = int32_t(e * nn + node_cols[a + t]);
    }
  if (rowptr) rowptr[nn * bs] = int32_t(nnz);
}

}  // namespace db2
