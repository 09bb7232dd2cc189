// capi.cpp -- the extern "C" boundary: status codes instead of exceptions,
// opaque handles, thread-local error messages.
#include <cuda_runtime.h>

#include <cstring>
#include <functional>
#include <memory>
#include <new>
#include <string>

#include "internal.h"

struct db2_mesh_t {
  std::shared_ptr<db2::Mesh> m;
};
struct db2_space_t {
  std::shared_ptr<db2::Space> V;
};
struct db2_pattern_t {
  std::shared_ptr<db2::Pattern> P;
  db2::DeviceBuffer scratch;  // adjoint work array (grown on demand)
};

namespace db2 {
int64_t launches();
ReorderedCSR& reordered_on_device(Pattern& P);
void gather_values(Pattern& P, double* vals, bool add, void* stream);
void gather_dofs(Pattern& P, double* dst, const double* src_nat, bool add, void* stream);
void scatter_dofs(Pattern& P, double* dst_nat, const double* src, void* stream);
void scatter_flags(Pattern& P, uint8_t* dst_nat, const uint8_t* src, void* stream);
void scatter_values(Pattern& P, double* dst_nat, const double* src, void* stream);
std::shared_ptr<Pattern> pattern_of(db2_pattern P) { return P ? P->P : nullptr; }
}

namespace {
thread_local std::string g_err;

template <typename F>
int guard(F&& f) {
  try {
    f();
    return DB2_OK;
  } catch (const db2::Error& e) {
    g_err = e.msg;
    return e.code;
  } catch (const std::bad_alloc&) {
    g_err = "host allocation failed";
    return DB2_ERR_NOMEM;
  } catch (const std::exception& e) {
    g_err = e.what();
    return DB2_ERR_ARGUMENT;
  } catch (...) {
    g_err = "unknown error";
    return DB2_ERR_ARGUMENT;
  }
}

void need(const void* p, const char* what) {
  if (!p) db2::fail(DB2_ERR_ARGUMENT, "%s is NULL", what);
}

db2::FormArgs form_args(const db2_form* f, const double* w) {
  db2::FormArgs a;
  a.f = *f;
  a.w = w;
  return a;
}
}  // namespace

namespace db2 {
int guard_call(const std::function<void()>& f) { return guard(f); }
}

extern "C" {

const char* db2_last_error(void) { return g_err.c_str(); }
const char* db2_version(void) { return "dolfin_b200 0.1 (sm_100a)"; }
int64_t db2_kernel_launches(void) { return db2::launches(); }

int db2_mesh_create(int tdim, int64_t nv, const double* coords, int64_t nc, const uint32_t* cells,
                    db2_mesh* out) {
  return guard([&] {
    need(out, "out");
    auto h = new db2_mesh_t{db2::make_mesh(tdim, nv, coords, nc, cells)};
    *out = h;
  });
}

int db2_mesh_unit_cube(int nx, int ny, int nz, db2_mesh* out) {
  return guard([&] {
    need(out, "out");
    *out = new db2_mesh_t{db2::make_unit_cube(nx, ny, nz)};
  });
}

int db2_mesh_unit_square(int nx, int ny, int diagonal, db2_mesh* out) {
  return guard([&] {
    need(out, "out");
    *out = new db2_mesh_t{db2::make_unit_square(nx, ny, diagonal)};
  });
}

int db2_mesh_info(db2_mesh m, int* tdim, int64_t* nv, int64_t* nc) {
  return guard([&] {
    need(m, "mesh");
    if (tdim) *tdim = m->m->tdim;
    if (nv) *nv = m->m->nv;
    if (nc) *nc = m->m->nc;
  });
}

int db2_mesh_copy(db2_mesh m, double* coords, uint32_t* cells) {
  return guard([&] {
    need(m, "mesh");
    if (coords) std::memcpy(coords, m->m->x.data(), m->m->x.size() * sizeof(double));
    if (cells) std::memcpy(cells, m->m->cells.data(), m->m->cells.size() * sizeof(uint32_t));
  });
}

int db2_mesh_set_coordinates(db2_mesh m, const double* coords) {
  return guard([&] {
    need(m, "mesh");
    need(coords, "coords");
    std::memcpy(m->m->x.data(), coords, m->m->x.size() * sizeof(double));
    if (m->m->on_device) m->m->upload_coordinates();
  });
}

int db2_mesh_num_edges(db2_mesh m, int64_t* ne) {
  return guard([&] {
    need(m, "mesh");
    need(ne, "ne");
    m->m->compute_edges();
    *ne = m->m->ne;
  });
}

int db2_mesh_num_exterior_facets(db2_mesh m, int64_t* n) {
  return guard([&] {
    need(m, "mesh");
    need(n, "n");
    m->m->compute_exterior_facets();
    *n = int64_t(m->m->ext_facets.size());
  });
}

int db2_mesh_exterior_facets(db2_mesh m, uint32_t* cell, int32_t* local_facet) {
  return guard([&] {
    need(m, "mesh");
    m->m->compute_exterior_facets();
    const auto& E = m->m->ext_facets;
    for (size_t i = 0; i < E.size(); ++i) {
      if (cell) cell[i] = E[i] >> 2;
      if (local_facet) local_facet[i] = int32_t(E[i] & 3u);
    }
  });
}

int db2_mesh_read_xml(const char* path, db2_mesh* out) {
  return guard([&] {
    need(path, "path");
    need(out, "out");
    *out = new db2_mesh_t{db2::read_mesh_xml(path)};
  });
}

int db2_mesh_write_xml(db2_mesh m, const char* path) {
  return guard([&] {
    need(m, "mesh");
    need(path, "path");
    db2::write_mesh_xml(*m->m, path);
  });
}

int db2_mesh_read_xdmf(const char* path, db2_mesh* out) {
  return guard([&] {
    need(path, "path");
    need(out, "out");
    *out = new db2_mesh_t{db2::read_mesh_xdmf(path)};
  });
}

int db2_mesh_write_xdmf(db2_mesh m, const char* path, const double* values, int value_size,
                        const char* name) {
  return guard([&] {
    need(m, "mesh");
    need(path, "path");
    db2::write_mesh_xdmf(*m->m, path, values, value_size, name);
  });
}

int db2_vector_write_xml(const char* path, int64_t n, const double* x) {
  return guard([&] {
    need(path, "path");
    need(x, "x");
    db2::write_vector_xml(path, n, x);
  });
}

int db2_vector_read_xml(const char* path, int64_t* n, double* x) {
  return guard([&] {
    need(path, "path");
    need(n, "n");
    *n = db2::read_vector_xml(path, x, *n);
  });
}

int db2_mesh_destroy(db2_mesh m) {
  delete m;
  return DB2_OK;
}

int db2_space_create(db2_mesh m, int degree, int value_size, db2_space* out) {
  return guard([&] {
    need(m, "mesh");
    need(out, "out");
    *out = new db2_space_t{db2::make_space(m->m, degree, value_size)};
  });
}

int db2_space_create_reordered(db2_mesh m, int degree, int value_size, db2_space* out) {
  return guard([&] {
    need(m, "mesh");
    need(out, "out");
    auto V = db2::make_space(m->m, degree, value_size);
    V->node_new = db2::rcm_node_order(*V);
    *out = new db2_space_t{V};
  });
}

int db2_space_node_numbers(db2_space V, int32_t* node_new) {
  return guard([&] {
    need(V, "space");
    need(node_new, "node_new");
    const auto& S = *V->V;
    for (int64_t i = 0; i < S.nnodes; ++i) node_new[i] = S.reordered() ? S.node_new[i] : int32_t(i);
  });
}

int db2_space_info(db2_space V, int* ndofs_per_cell, int64_t* dim) {
  return guard([&] {
    need(V, "space");
    if (ndofs_per_cell) *ndofs_per_cell = V->V->k * V->V->vsize;
    if (dim) *dim = V->V->dim();
  });
}

// DofMap::cell_dofs: component-major local order, dof = c*nnodes + node.
int db2_space_cell_dofs(db2_space V, int32_t* out) {
  return guard([&] {
    need(V, "space");
    need(out, "out");
    const auto& S = *V->V;
    const int k = S.k, n = k * S.vsize;
    for (int64_t c = 0; c < S.mesh->nc; ++c)
      for (int comp = 0; comp < S.vsize; ++comp)
        for (int i = 0; i < k; ++i)
          out[c * n + comp * k + i] = int32_t(S.dof(comp, S.cell_nodes[c * k + i]));
  });
}

int db2_space_destroy(db2_space V) {
  delete V;
  return DB2_OK;
}

int db2_pattern_create(db2_space V, int keep_diagonal, db2_pattern* out) {
  return guard([&] {
    need(V, "space");
    need(out, "out");
    auto h = new db2_pattern_t;
    try {
      h->P = db2::make_pattern(V->V, keep_diagonal != 0);
    } catch (...) {
      delete h;
      throw;
    }
    *out = h;
  });
}

int db2_pattern_info(db2_pattern P, int64_t* nrows, int64_t* nnz) {
  return guard([&] {
    need(P, "pattern");
    if (nrows) *nrows = P->P->nrows;
    if (nnz) *nnz = P->P->nnz;
  });
}

int db2_pattern_csr_device(db2_pattern P, const int32_t** rowptr, const int32_t** cols) {
  return guard([&] {
    need(P, "pattern");
    P->P->ensure_device();
    if (P->P->V->reordered()) {
      db2::ReorderedCSR& R = db2::reordered_on_device(*P->P);
      if (rowptr) *rowptr = R.d_rowptr.as<int32_t>();
      if (cols) *cols = R.d_cols.as<int32_t>();
      return;
    }
    if (rowptr) *rowptr = P->P->d_rowptr.as<int32_t>();
    if (cols) *cols = P->P->d_cols.as<int32_t>();
  });
}

int db2_pattern_csr_host(db2_pattern P, int32_t* rowptr, int32_t* cols) {
  return guard([&] {
    need(P, "pattern");
    P->P->csr_host(rowptr, cols);
  });
}

int db2_pattern_plan_info(db2_pattern P, int64_t* nnodes, int64_t* nincidences, int* kp,
                          int64_t* ntiles, int64_t* ngroups, int64_t* ntypes) {
  return guard([&] {
    need(P, "pattern");
    if (nnodes) *nnodes = P->P->V->nnodes;
    if (nincidences) *nincidences = int64_t(P->P->inc.size());
    if (kp) *kp = P->P->kp;
    if (ntiles) *ntiles = int64_t(P->P->tiles.size());
    if (ngroups) *ngroups = 0;
    if (ntypes) *ntypes = 0;
  });
}

int db2_pattern_plan_copy(db2_pattern P, int32_t* node_rowptr, int32_t* node_cols,
                          uint32_t* inc_ptr, uint32_t* inc, uint8_t* pos, int32_t* tiles) {
  return guard([&] {
    need(P, "pattern");
    const auto& Q = *P->P;
    if (node_rowptr) std::memcpy(node_rowptr, Q.node_rowptr.data(), Q.node_rowptr.size() * 4);
    if (node_cols) std::memcpy(node_cols, Q.node_cols.data(), Q.node_cols.size() * 4);
    if (inc_ptr) std::memcpy(inc_ptr, Q.inc_ptr.data(), Q.inc_ptr.size() * 4);
    if (inc) std::memcpy(inc, Q.inc.data(), Q.inc.size() * 4);
    if (pos) std::memcpy(pos, Q.pos.data(), Q.pos.size());
    if (tiles) std::memcpy(tiles, Q.tiles.data(), Q.tiles.size() * sizeof(db2::Tile));
  });
}

int db2_pattern_retile(db2_pattern P, int tile_threads, int seg_cap_bytes) {
  return guard([&] {
    need(P, "pattern");
    db2::retile(*P->P, tile_threads, seg_cap_bytes);
  });
}

int db2_pattern_set_row_range(db2_pattern P, int64_t node_begin, int64_t node_end) {
  return guard([&] {
    need(P, "pattern");
    db2::set_row_range(*P->P, node_begin, node_end);
  });
}

int db2_pattern_set_row_block(db2_pattern P, int64_t node_begin, int64_t node_end) {
  return guard([&] {
    need(P, "pattern");
    db2::set_row_range(*P->P, node_begin, node_end, true);
  });
}

int db2_pattern_row_block_info(db2_pattern P, int64_t* nrows, int64_t* nnz) {
  return guard([&] {
    need(P, "pattern");
    db2::row_block_size(*P->P, nrows, nnz);
  });
}

int db2_pattern_row_block_csr_host(db2_pattern P, int32_t* rowptr, int32_t* cols) {
  return guard([&] {
    need(P, "pattern");
    const db2::Pattern& Q = *P->P;
    if (Q.V->reordered()) db2::fail(DB2_ERR_UNSUPPORTED, "row blocks are provided for the natural numbering");
    const int64_t nn = Q.V->nnodes, n0 = Q.row_begin, n1 = Q.row_end < 0 ? nn : Q.row_end;
    const int bs = Q.bs;
    int64_t at = 0, r = 0;
    for (int c = 0; c < bs; ++c)
      for (int64_t i = n0; i < n1; ++i, ++r) {
        const int32_t a = Q.node_rowptr[i], L = Q.node_rowptr[i + 1] - a;
        if (rowptr) rowptr[r] = int32_t(at);
        if (cols)
          for (int e = 0; e < bs; ++e)
            for (int32_t t = 0; t < L; ++t) cols[at + int64_t(e) * L + t] = int32_t(e * nn + Q.node_cols[a + t]);
        at += int64_t(bs) * L;
      }
    if (rowptr) rowptr[r] = int32_t(at);
  });
}

int db2_pattern_facet_plan_info(db2_pattern P, int64_t* nbnodes, int64_t* nincidences, int* kf) {
  return guard([&] {
    need(P, "pattern");
    db2::build_facet_plan(*P->P);
    const db2::FacetPlan& F = *P->P->facets;
    if (nbnodes) *nbnodes = int64_t(F.bnode.size());
    if (nincidences) *nincidences = int64_t(F.binc_ptr.back());
    if (kf) *kf = F.kf;
  });
}

int db2_pattern_facet_plan_copy(db2_pattern P, uint32_t* bnode, uint32_t* binc_ptr,
                                uint32_t* bverts, uint8_t* bslot) {
  return guard([&] {
    need(P, "pattern");
    db2::build_facet_plan(*P->P);
    const db2::FacetPlan& F = *P->P->facets;
    auto cp = [](auto* dst, const auto& v) {
      if (dst) std::memcpy(dst, v.data(), v.size() * sizeof(v[0]));
    };
    cp(bnode, F.bnode);
    cp(binc_ptr, F.binc_ptr);
    cp(bverts, F.bverts);
    cp(bslot, F.bslot);
  });
}

int db2_pattern_destroy(db2_pattern P) {
  delete P;
  return DB2_OK;
}

int db2_assemble_matrix(db2_pattern P, const db2_form* a, const double* w, int precision,
                        double* vals, int add_values, void* stream) {
  return guard([&] {
    need(P, "pattern");
    need(a, "form");
    need(vals, "vals");
    const db2::FormArgs fa = form_args(a, w);
    db2::Pattern& Pt = *P->P;
    // reordered space: assemble in natural order into scratch, then gather
    const bool ro = Pt.V->reordered();
    double* out = ro ? db2::reordered_on_device(Pt).d_vals.as<double>() : vals;
    const bool add = ro ? false : add_values != 0;
    if (a->kind == DB2_FORM_FACET_MASS)
      db2::launch_facet_matrix(Pt, fa, out, add, nullptr, nullptr, nullptr, stream);
    else
      db2::launch_assemble(Pt, &fa, nullptr, precision, out, nullptr, add, nullptr, nullptr, stream);
    if (ro) db2::gather_values(Pt, vals, add_values != 0, stream);
  });
}

int db2_assemble_vector(db2_pattern P, const db2_form* L, const double* w, double* b,
                        int add_values, void* stream) {
  return guard([&] {
    need(P, "pattern");
    need(L, "form");
    need(b, "b");
    const db2::FormArgs fl = form_args(L, w);
    db2::Pattern& Pt = *P->P;
    const bool ro = Pt.V->reordered();
    double* out = ro ? db2::reordered_on_device(Pt).d_b.as<double>() : b;
    const bool add = ro ? false : add_values != 0;
    if (L->kind == DB2_FORM_FACET_LOAD)
      db2::launch_facet_vector(Pt, fl, out, add, nullptr, stream);
    else
      db2::launch_assemble(Pt, nullptr, &fl, DB2_FP64, nullptr, out, add, nullptr, nullptr, stream);
    if (ro) db2::gather_dofs(Pt, b, out, add_values != 0, stream);
  });
}

int db2_assemble_scalar(db2_mesh m, const db2_form* M, const double* w, double* out,
                        void* stream) {
  return guard([&] {
    need(m, "mesh");
    need(M, "form");
    need(out, "out");
    db2::launch_functional(*m->m, form_args(M, w), out, stream);
  });
}

int db2_assemble_local(db2_space V, const db2_form* a, const double* w, const db2_form* a_ds,
                       const double* w_ds, int64_t ncells, const uint32_t* cells, double* out,
                       void* stream) {
  return guard([&] {
    need(V, "space");
    need(cells, "cells");
    need(out, "out");
    db2::FormArgs fa, fd;
    if (a) fa = form_args(a, w);
    if (a_ds) fd = form_args(a_ds, w_ds);
    db2::launch_local(*V->V, a ? &fa : nullptr, a_ds ? &fd : nullptr, ncells, cells, out, stream);
  });
}

int db2_assemble_facets_bc(db2_pattern P, const db2_form* a_ds, const double* wa,
                           const db2_form* L_ds, const double* wL, const uint8_t* bc_flags,
                           const double* bc_vals, double* vals, double* b, void* stream) {
  return guard([&] {
    need(P, "pattern");
    need(bc_flags, "bc_flags");
    need(bc_vals, "bc_vals");
    need(b, "b");
    db2::Pattern& Pt = *P->P;
    if (a_ds) need(vals, "vals");
    if (Pt.V->reordered()) {
      // natural scratch from zero, the facet terms added there, then gathered
      // and added to the caller's arrays
      db2::ReorderedCSR& R = db2::reordered_on_device(Pt);
      cudaStream_t s = static_cast<cudaStream_t>(stream);
      db2::scatter_flags(Pt, R.d_flags.as<uint8_t>(), bc_flags, stream);
      db2::scatter_dofs(Pt, R.d_bcv.as<double>(), bc_vals, stream);
      cudaMemsetAsync(R.d_b.ptr, 0, size_t(Pt.V->dim()) * sizeof(double), s);
      if (a_ds) {
        cudaMemsetAsync(R.d_vals.ptr, 0, size_t(Pt.nnz) * sizeof(double), s);
        db2::launch_facet_matrix(Pt, form_args(a_ds, wa), R.d_vals.as<double>(), true,
                                 R.d_flags.as<uint8_t>(), R.d_bcv.as<double>(), R.d_b.as<double>(), stream);
        db2::gather_values(Pt, vals, true, stream);
      }
      if (L_ds)
        db2::launch_facet_vector(Pt, form_args(L_ds, wL), R.d_b.as<double>(), true,
                                 R.d_flags.as<uint8_t>(), stream);
      db2::gather_dofs(Pt, b, R.d_b.as<double>(), true, stream);
      return;
    }
    if (a_ds) db2::launch_facet_matrix(Pt, form_args(a_ds, wa), vals, true, bc_flags, bc_vals, b, stream);
    if (L_ds) db2::launch_facet_vector(Pt, form_args(L_ds, wL), b, true, bc_flags, stream);
  });
}

int db2_assemble_system(db2_pattern P, const db2_form* a, const double* wa, const db2_form* L,
                        const double* wL, int precision, double* vals, double* b, void* stream) {
  return guard([&] {
    need(P, "pattern");
    need(a, "bilinear form");
    need(L, "linear form");
    need(vals, "vals");
    need(b, "b");
    const db2::FormArgs fa = form_args(a, wa), fl = form_args(L, wL);
    db2::Pattern& Pt = *P->P;
    if (Pt.V->reordered()) {
      db2::ReorderedCSR& R = db2::reordered_on_device(Pt);
      db2::launch_assemble(Pt, &fa, &fl, precision, R.d_vals.as<double>(), R.d_b.as<double>(), false,
                           nullptr, nullptr, stream);
      db2::gather_values(Pt, vals, false, stream);
      db2::gather_dofs(Pt, b, R.d_b.as<double>(), false, stream);
      return;
    }
    db2::launch_assemble(Pt, &fa, &fl, precision, vals, b, false, nullptr, nullptr, stream);
  });
}

int db2_assemble_system_bc(db2_pattern P, const db2_form* a, const double* wa, const db2_form* L,
                           const double* wL, const uint8_t* bc_flags, const double* bc_vals,
                           int precision, double* vals, double* b, void* stream) {
  return guard([&] {
    need(P, "pattern");
    need(a, "bilinear form");
    need(L, "linear form");
    need(bc_flags, "bc_flags");
    need(bc_vals, "bc_vals");
    const db2::FormArgs fa = form_args(a, wa), fl = form_args(L, wL);
    db2::Pattern& Pt = *P->P;
    if (Pt.V->reordered()) {
      db2::ReorderedCSR& R = db2::reordered_on_device(Pt);
      db2::scatter_flags(Pt, R.d_flags.as<uint8_t>(), bc_flags, stream);
      db2::scatter_dofs(Pt, R.d_bcv.as<double>(), bc_vals, stream);
      db2::launch_assemble(Pt, &fa, &fl, precision, R.d_vals.as<double>(), R.d_b.as<double>(), false,
                           R.d_flags.as<uint8_t>(), R.d_bcv.as<double>(), stream);
      db2::gather_values(Pt, vals, false, stream);
      db2::gather_dofs(Pt, b, R.d_b.as<double>(), false, stream);
      return;
    }
    db2::launch_assemble(Pt, &fa, &fl, precision, vals, b, false, bc_flags, bc_vals, stream);
  });
}

int db2_apply(db2_pattern P, const db2_form* a, const double* w, int precision, const double* x,
              double* y, void* stream) {
  return guard([&] {
    need(P, "pattern");
    need(a, "form");
    need(x, "x");
    need(y, "y");
    db2::Pattern& Pt = *P->P;
    if (Pt.V->reordered()) {
      db2::ReorderedCSR& R = db2::reordered_on_device(Pt);
      db2::scatter_dofs(Pt, R.d_vec.as<double>(), x, stream);
      db2::launch_apply(Pt, form_args(a, w), precision, R.d_vec.as<double>(), R.d_b.as<double>(), stream);
      db2::gather_dofs(Pt, y, R.d_b.as<double>(), false, stream);
      return;
    }
    db2::launch_apply(Pt, form_args(a, w), precision, x, y, stream);
  });
}

int db2_tensor_core_status(int* status) {
  return guard([&] {
    need(status, "status");
    *status = db2::tensor_core_status();
  });
}

int db2_vjp_kappa(db2_pattern P, const db2_form* a, const double* kappa, const db2_form* L,
                  const double* f, const double* gA, const double* gb, int precision,
                  double* dkappa, void* stream) {
  return guard([&] {
    need(P, "pattern");
    need(a, "form");
    need(kappa, "kappa");
    need(gA, "gA");
    need(dkappa, "dkappa");
    const size_t need_d = db2::vjp_scratch_doubles(*P->P);
    if (P->scratch.bytes < need_d * sizeof(double)) P->scratch.alloc(need_d * sizeof(double));
    db2::FormArgs fl;
    if (L) fl = form_args(L, f);
    else {
      std::memset(&fl.f, 0, sizeof(fl.f));
      fl.f.kind = DB2_FORM_LOAD;
      fl.f.coeff = DB2_COEFF_NONE;
    }
    db2::Pattern& Pt = *P->P;
    if (Pt.block_storage)
      db2::fail(DB2_ERR_UNSUPPORTED, "the adjoint takes whole-CSR gradients (no row-block storage)");
    if (Pt.V->reordered()) {
      // upstream gradients into the natural numbering
      db2::ReorderedCSR& R = db2::reordered_on_device(Pt);
      db2::scatter_values(Pt, R.d_vals.as<double>(), gA, stream);
      if (L && gb) db2::scatter_dofs(Pt, R.d_b.as<double>(), gb, stream);
      gA = R.d_vals.as<double>();
      if (L && gb) gb = R.d_b.as<double>();
    }
    db2::launch_vjp(Pt, form_args(a, kappa), fl, precision, gA, L ? gb : nullptr, dkappa,
                    P->scratch.as<double>(), stream);
  });
}

}  // extern "C"
