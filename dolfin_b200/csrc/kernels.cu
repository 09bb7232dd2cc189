// kernels.cu -- launchers of the assembly, vector, action and adjoint kernels.
#include <cuda_runtime.h>

#include "launch.cuh"

namespace db2 {

namespace dev {

// Vector-only assembly (Assembler::assemble for a rank-1 form): one thread
// per dof (component c, node i) gathering its incident cells in cell order.
template <int D, int P, int LOADM>
__global__ void __launch_bounds__(256) k_assemble_vector(const AsmParams p, int bs, int64_t n0,
                                                         int64_t nrange) {
  const int64_t r = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (r >= nrange * bs) return;
  const int c = int(r / nrange);
  const int64_t node = n0 + (r - int64_t(c) * nrange);
  double bsum = 0.0;
  const uint32_t i0 = __ldg(p.inc_ptr + node);
  const uint32_t cnt = __ldg(p.inc_ptr + node + 1) - i0;
  const uint32_t rbase = __ldg(p.rec_goff + (node >> 5)) + uint32_t(node & 31);
  const RowFix<D> F = load_row_fix<D, P, LOADM == LOAD_P1>(p, uint32_t(node));
  for (uint32_t m = 0; m < cnt; ++m) {
    const Rec<D, P> r = load_rec<D, P>(p, rbase + 32u * m);
    double x[D + 1][D], kap[D + 1], fv[D + 1];
    record_cell<D, P, LOADM == LOAD_P1>(p, F, r, i0 + m, x, kap, fv);
    Geometry<D> G;
    geometry(x, G);
    bsum += load_row<D, P, LOADM>(p, G, F.nfix == 1, c, fv, kap);
  }
  double* bp = p.b + int64_t(c) * p.bstride + node - p.bbase;
  *bp = p.add_values ? *bp + bsum : bsum;
}

// Vertex records for one call: the w slots of (x, y, z, w) carry kappa (3D);
// 2D records are (x, y, kappa, f).
__global__ void k_pack_vertex_records(double* __restrict__ xw, int64_t nv, int tdim,
                                      const double* __restrict__ kappa,
                                      const double* __restrict__ f) {
  const int64_t v = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (v >= nv) return;
  if (tdim == 3) {
    xw[4 * v + 3] = kappa ? kappa[v] : 0.0;
  } else {
    xw[4 * v + 2] = kappa ? kappa[v] : 0.0;
    xw[4 * v + 3] = f ? f[v] : 0.0;
  }
}

}  // namespace dev

// Writes kappa (and f in 2D) into the mesh's vertex records on `stream`.
void pack_vertex_records(const Pattern& P, const double* kappa, const double* f, void* stream) {
  const Mesh& m = *P.V->mesh;
  if (!kappa && !(m.tdim == 2 && f)) return;
  const int threads = 256;
  dev::k_pack_vertex_records<<<unsigned((m.nv + threads - 1) / threads), threads, 0,
                               static_cast<cudaStream_t>(stream)>>>(
      m.d_x.as<double>(), m.nv, m.tdim, kappa, f);
  count_launch();
  check_cuda("pack_vertex_records launch");
}

dev::AsmParams make_params(const Pattern& P) {
  const_cast<Pattern&>(P).ensure_device();
  dev::AsmParams p{};
  const Mesh& m = *P.V->mesh;
  p.tiles = P.d_tiles.as<Tile>();
  p.node_rowptr = P.d_node_rowptr.as<int32_t>();
  p.inc_ptr = P.d_inc_ptr.as<uint32_t>();
  p.rec = P.d_rec.as<unsigned char>();
  p.rec_goff = P.d_rec_goff.as<uint32_t>();
  p.rec_first = P.d_rec_first.as<unsigned char>();
  p.inc = P.d_inc.as<uint32_t>();
  p.cols = P.d_cols.as<int32_t>();
  p.edge_v = P.V->d_edge_vertices.as<uint32_t>();
  p.nverts = m.nv;
  p.cells = m.d_cells.as<uint32_t>();
  p.xw = m.d_x.as<double>();
  p.cell_nodes = P.V->d_cell_nodes.as<uint32_t>();
  p.cell_inc = P.d_cell_inc.as<uint32_t>();
  p.kscale = 1.0;
  p.fc[0] = p.fc[1] = p.fc[2] = 0.0;
  p.nnz_node = P.nnz_node;
  p.nnodes = P.V->nnodes;
  const OutputLayout o = output_layout(P);
  p.vstride = o.vstride;
  p.vbase = o.vbase;
  p.bstride = o.bstride;
  p.bbase = o.bbase;
  return p;
}

// kappa of a bilinear form -> (uses P1 field, scale)
static bool matrix_coeff(const FormArgs& a, dev::AsmParams& p) {
  switch (a.f.coeff) {
    case DB2_COEFF_NONE: p.kscale = 1.0; return false;
    case DB2_COEFF_CONSTANT: p.kscale = a.f.constant[0]; return false;
    case DB2_COEFF_P1:
    case DB2_COEFF_P1_SCALED:
      if (!a.w) fail(DB2_ERR_ARGUMENT, "form coefficient is a P1 Function but no field was given");
      p.kappa = a.w;
      p.kscale = a.f.coeff == DB2_COEFF_P1 ? 1.0 : a.f.constant[0];
      return true;
    default: fail(DB2_ERR_ARGUMENT, "unknown coefficient kind %d", a.f.coeff);
  }
}

static int load_mode(const FormArgs* L, int bs, dev::AsmParams& p) {
  if (!L) return dev::LOAD_NONE;
  if (L->f.kind != DB2_FORM_LOAD) fail(DB2_ERR_ARGUMENT, "linear form must be DB2_FORM_LOAD");
  switch (L->f.coeff) {
    case DB2_COEFF_NONE:
      for (int c = 0; c < 3; ++c) p.fc[c] = 1.0;
      return dev::LOAD_CONST;
    case DB2_COEFF_CONSTANT:
      for (int c = 0; c < 3; ++c) p.fc[c] = bs == 1 ? L->f.constant[0] : L->f.constant[c];
      return dev::LOAD_CONST;
    case DB2_COEFF_P1:
    case DB2_COEFF_P1_SCALED:
      if (bs != 1) fail(DB2_ERR_UNSUPPORTED, "P1 load coefficient on a vector space");
      if (!L->w) fail(DB2_ERR_ARGUMENT, "load coefficient is a P1 Function but no field was given");
      p.f = L->w;
      p.fc[0] = L->f.coeff == DB2_COEFF_P1 ? 1.0 : L->f.constant[0];
      return dev::LOAD_P1;
    case DB2_COEFF_P1_KAPPA:
      if (bs != 1) fail(DB2_ERR_UNSUPPORTED, "kappa-weighted load on a vector space");
      if (!L->w) fail(DB2_ERR_ARGUMENT, "kappa-weighted load: no field f was given");
      p.f = L->w;
      p.fc[0] = L->f.constant[0];
      return dev::LOAD_KP1;
    default: fail(DB2_ERR_ARGUMENT, "unknown coefficient kind %d", L->f.coeff);
  }
}

void launch_assemble(const Pattern& P, const FormArgs* a, const FormArgs* L, int precision,
                     double* vals, double* b, bool add_values, const uint8_t* bc_flags,
                     const double* bc_vals, void* stream) {
  const Space& V = *P.V;
  const int D = V.mesh->tdim;
  // the tile kernel writes its value segments with 16-byte bulk copies from
  // an 8-byte-aligned base (and doubles elsewhere): refuse other pointers
  // here rather than fault on the device
  if ((reinterpret_cast<uintptr_t>(vals) | reinterpret_cast<uintptr_t>(b)) % alignof(double))
    fail(DB2_ERR_ARGUMENT, "value and vector arrays must be 8-byte aligned device pointers");
  dev::AsmParams p = make_params(P);
  p.vals = vals;
  p.b = b;
  p.add_values = add_values ? 1 : 0;
  p.bc_flags = bc_flags;
  p.bc_vals = bc_vals;
  const int loadm = load_mode(L, P.bs, p);
  if (loadm == dev::LOAD_KP1 && !(a && a->f.kind == DB2_FORM_DIFFUSION &&
                                  (a->f.coeff == DB2_COEFF_P1 || a->f.coeff == DB2_COEFF_P1_SCALED)))
    fail(DB2_ERR_UNSUPPORTED, "a kappa-weighted load (DB2_COEFF_P1_KAPPA) is assembled together with "
         "kappa*grad(u).grad(v)*dx with a P1 kappa (db2_assemble_system / _system_bc)");
  if (!a) {
    pack_vertex_records(P, nullptr, loadm == dev::LOAD_P1 ? p.f : nullptr, stream);
    // rank-1 form only
    if (loadm == dev::LOAD_NONE) fail(DB2_ERR_ARGUMENT, "nothing to assemble");
    // the node rows of the pattern's row range (all of them by default)
    const int64_t n0 = P.row_begin, nr = (P.row_end < 0 ? V.nnodes : P.row_end) - n0;
    const int64_t n = nr * P.bs;
    if (n == 0) return;
    const int threads = 256;
    const unsigned blocks = unsigned((n + threads - 1) / threads);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
#define DB2_VEC(D_, P_)                                                                       \
  if (D == D_ && V.degree == P_) {                                                            \
    if (loadm == dev::LOAD_CONST) dev::k_assemble_vector<D_, P_, dev::LOAD_CONST><<<blocks, threads, 0, s>>>(p, P.bs, n0, nr); \
    else dev::k_assemble_vector<D_, P_, dev::LOAD_P1><<<blocks, threads, 0, s>>>(p, P.bs, n0, nr);    \
    count_launch();                                                                           \
    check_cuda("assemble_vector launch");                                                     \
    return;                                                                                   \
  }
    DB2_VEC(3, 1) DB2_VEC(3, 2) DB2_VEC(2, 1) DB2_VEC(2, 2)
#undef DB2_VEC
    fail(DB2_ERR_UNSUPPORTED, "vector assembly not provided for this element");
  }
  if (bc_flags && (!bc_vals || !L || !b)) fail(DB2_ERR_ARGUMENT, "Dirichlet data needs values, a linear form and b");
  p.cols = P.d_cols.as<int32_t>();
  dev::LaunchCfg cfg;
  cfg.class_begin = &P.class_begin;
  cfg.class_smem = &P.class_smem;
  cfg.threads = P.tile_threads;
  cfg.stream = static_cast<cudaStream_t>(stream);
  cfg.escapes = P.rec_escapes > 0;
  const bool fp32 = precision == DB2_FP32_CONTRACT;
  if (precision != DB2_FP64 && precision != DB2_FP32_CONTRACT) fail(DB2_ERR_ARGUMENT, "unknown precision %d", precision);
  bool ok = false;
  if (a->f.kind == DB2_FORM_DIFFUSION) {
    if (P.bs != 1) fail(DB2_ERR_UNSUPPORTED, "diffusion form on a vector space");
    const bool kp1 = matrix_coeff(*a, p);
    pack_vertex_records(P, kp1 ? p.kappa : nullptr,
                        (loadm == dev::LOAD_P1 || loadm == dev::LOAD_KP1) ? p.f : nullptr, stream);
    ok = D == 3 ? dev::dispatch_tet_diff(V.degree, p, cfg, kp1, loadm, fp32)
                : dev::dispatch_tri_diff(V.degree, p, cfg, kp1, loadm, fp32);
  } else if (a->f.kind == DB2_FORM_ELASTICITY) {
    if (P.bs != D || D != 3) fail(DB2_ERR_UNSUPPORTED, "elasticity needs a 3D vector space");
    p.mu = a->f.mu;
    p.lmbda = a->f.lmbda;
    if (a->f.coeff != DB2_COEFF_NONE) fail(DB2_ERR_UNSUPPORTED, "elasticity takes no coefficient");
    pack_vertex_records(P, nullptr, nullptr, stream);
    ok = dev::dispatch_tet_elas(V.degree, p, cfg, false, loadm, fp32);
  } else {
    fail(DB2_ERR_ARGUMENT, "bilinear form kind %d not provided", a->f.kind);
  }
  if (!ok) fail(DB2_ERR_UNSUPPORTED, "no kernel for this form/coefficient/load combination");
}

}  // namespace db2
