// facets.cu -- exterior-facet integrals (ds) and functionals (rank-0 forms).
//
// Replaces Assembler::assemble_exterior_facets (dolfin/fem/Assembler.cpp:
// 196-288) for the forms
//     a = w * u * v * ds      (Robin / boundary mass, scalar P1/P2)
//     L = w * v * ds          (Neumann load, scalar P1/P2)
//     L = inner(t, v) * ds    (constant traction, vector P1/P2)
// with w = 1, a Constant or a P1 Function, and the functional assemble(M),
// double assemble(const Form&) (dolfin/fem/assemble.h:66), for
//     M = w * dx,  M = w * ds  (w = Constant, P1 Function or x[i]).
//
// Vector and matrix: one thread per boundary node walks that node's exterior
// facets in facet-number order (the order of the reference's facet loop) and
// adds into its own entries of b or of its own CSR row -- no two threads
// write the same address, so the result is deterministic without atomics.
// These run after the cell pass on the same stream and add to its output.
// Functionals: a fixed grid walks the cells / facets with a fixed stride and
// reduces in a fixed tree, then one block sums the per-block partials: the
// same summation order on every run.
#include <cuda_runtime.h>

#include <algorithm>

#include "facet_rows.cuh"

namespace db2 {
namespace dev {

struct FacetParams {
  const uint32_t* bnode;
  const uint32_t* binc_ptr;
  const uint32_t* bverts;
  const uint8_t* bslot;
  const double* xw;          // 4 doubles per vertex, coordinates first
  const double* w;           // P1 coefficient (vertex values) or null
  double scale;              // constant factor of the form
  double t[3];               // traction components (vector load)
  const int32_t* rowptr;     // scalar CSR (matrix)
  const int32_t* cols;
  double* vals;
  double* b;
  const uint8_t* bc_flags;   // dof-level Dirichlet flags or null
  const double* bc_vals;
  int64_t nnodes, nverts;
  // boundary nodes handled by this launch: bnode[bn0 .. bn0 + nbnodes), the
  // ones inside the pattern's row range
  int64_t bn0, nbnodes;
  // output layout of the pattern (full arrays or a rank's row block)
  int64_t vbase, bstride, bbase;
  int bs;
};

template <int D>
__device__ __forceinline__ void load_facet(const FacetParams& p, uint32_t s, bool wp1,
                                           double (&x)[D][D], double (&w)[D]) {
#pragma unroll
  for (int a = 0; a < D; ++a) {
    const uint32_t v = __ldg(p.bverts + size_t(s) * D + a);
#pragma unroll
    for (int r = 0; r < D; ++r) x[a][r] = __ldg(p.xw + 4 * size_t(v) + r);
    w[a] = wp1 ? __ldg(p.w + v) : 0.0;
  }
}

// b[(c, node)] += t_c (or scale) * sum over the node's exterior facets F of
// |F| * row, Dirichlet rows excepted (their b entry is the boundary value).
template <int D, int P, bool WP1>
__global__ void __launch_bounds__(256) k_facet_vector(const FacetParams p) {
  const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= p.nbnodes) return;
  const int64_t t = p.bn0 + i;
  const uint32_t node = __ldg(p.bnode + t);
  const bool vertex = P == 1 || node < p.nverts;
  double acc = 0.0;
  const uint32_t s1 = __ldg(p.binc_ptr + t + 1);
  for (uint32_t s = __ldg(p.binc_ptr + t); s < s1; ++s) {
    double x[D][D], w[D];
    load_facet<D>(p, s, WP1, x, w);
    acc = fma(facet_measure<D>(x), facet_load_row<D, P, WP1>(vertex, w), acc);
  }
  for (int c = 0; c < p.bs; ++c) {
    const int64_t dof = int64_t(c) * p.nnodes + node;
    if (p.bc_flags && __ldg(p.bc_flags + dof)) continue;
    p.b[int64_t(c) * p.bstride + node - p.bbase] += (p.bs == 1 ? p.scale : p.t[c]) * acc;
  }
}

// Row `node` of the boundary mass: vals[row, slot] += scale |F| row_j for the
// facet nodes j of each exterior facet of the node.  With Dirichlet data
// (SystemAssembler::apply_bc, dolfin/fem/SystemAssembler.cpp:1037-1070, on the
// facet part of the cell tensor): a Dirichlet row takes nothing (the cell
// pass already set it); a Dirichlet column moves to b (b_i -= A_ij g_j).
template <int D, int P, bool WP1>
__global__ void __launch_bounds__(256) k_facet_matrix(const FacetParams p) {
  constexpr int KF = FacetRows<D, P>::KF;
  const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= p.nbnodes) return;
  const int64_t t = p.bn0 + i;
  const uint32_t node = __ldg(p.bnode + t);
  if (p.bc_flags && __ldg(p.bc_flags + node)) return;
  const bool vertex = P == 1 || node < p.nverts;
  const int32_t ra = __ldg(p.rowptr + node);
  double* row = p.vals + ra - p.vbase;
  double bsub = 0.0;
  const uint32_t s1 = __ldg(p.binc_ptr + t + 1);
  for (uint32_t s = __ldg(p.binc_ptr + t); s < s1; ++s) {
    double x[D][D], w[D];
    load_facet<D>(p, s, WP1, x, w);
    const double f = p.scale * facet_measure<D>(x);
    double o[KF];
    facet_mass_row<D, P, WP1>(vertex, w, o);
    const uint2 sl = __ldg(reinterpret_cast<const uint2*>(p.bslot) + s);
#pragma unroll
    for (int j = 0; j < KF; ++j) {
      const uint32_t slot = ((j < 4 ? sl.x : sl.y) >> (8 * (j & 3))) & 0xffu;
      const double v = f * o[j];
      if (p.bc_flags) {
        const int32_t col = __ldg(p.cols + ra + slot);
        if (__ldg(p.bc_flags + col)) {
          bsub = fma(v, __ldg(p.bc_vals + col), bsub);
          continue;
        }
      }
      row[slot] += v;
    }
  }
  if (p.bc_flags && bsub != 0.0) p.b[node - p.bbase] -= bsub;
}

// ---- functionals ------------------------------------------------------------
constexpr int kFunctionalBlocks = 512;
constexpr int kFunctionalThreads = 256;

enum { FN_ONE = 0, FN_P1 = 1, FN_COORD = 2 };

template <int D>
__device__ __forceinline__ double cell_measure(const double (&x)[D + 1][D]) {
  if constexpr (D == 2) {
    const double det = (x[1][0] - x[0][0]) * (x[2][1] - x[0][1]) -
                       (x[1][1] - x[0][1]) * (x[2][0] - x[0][0]);
    return 0.5 * fabs(det);
  } else {
    double c[3][3];
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int r = 0; r < 3; ++r) c[a][r] = x[a + 1][r] - x[0][r];
    const double det = c[0][0] * (c[1][1] * c[2][2] - c[1][2] * c[2][1]) -
                       c[0][1] * (c[1][0] * c[2][2] - c[1][2] * c[2][0]) +
                       c[0][2] * (c[1][0] * c[2][1] - c[1][1] * c[2][0]);
    return fabs(det) * (1.0 / 6.0);
  }
}

// One partial sum per block: item i of n (a cell, or an exterior facet)
// contributes |K| * mean of the integrand's vertex values (exact for P1).
template <int D, bool FACET>
__global__ void __launch_bounds__(kFunctionalThreads) k_functional(
    const double* __restrict__ xw, const uint32_t* __restrict__ cells,
    const uint32_t* __restrict__ ext, int64_t n, int mode, const double* __restrict__ w, int comp,
    double* __restrict__ partials) {
  constexpr int NV = FACET ? D : D + 1;
  __shared__ double red[kFunctionalThreads];
  double acc = 0.0;
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += int64_t(gridDim.x) * blockDim.x) {
    uint32_t v[NV];
    if constexpr (FACET) {
      const uint32_t e = __ldg(ext + i), c = e >> 2, fl = e & 3u;
      int m = 0;
#pragma unroll
      for (int a = 0; a <= D; ++a) {
        const uint32_t va = __ldg(cells + size_t(c) * (D + 1) + a);
        if (a != int(fl) && m < NV) v[m++] = va;
      }
    } else {
#pragma unroll
      for (int a = 0; a < NV; ++a) v[a] = __ldg(cells + size_t(i) * (D + 1) + a);
    }
    double meas, mean = 1.0;
    if constexpr (FACET) {
      double x[D][D];
#pragma unroll
      for (int a = 0; a < D; ++a)
#pragma unroll
        for (int r = 0; r < D; ++r) x[a][r] = __ldg(xw + 4 * size_t(v[a]) + r);
      meas = facet_measure<D>(x);
    } else {
      double x[D + 1][D];
#pragma unroll
      for (int a = 0; a <= D; ++a)
#pragma unroll
        for (int r = 0; r < D; ++r) x[a][r] = __ldg(xw + 4 * size_t(v[a]) + r);
      meas = cell_measure<D>(x);
    }
    if (mode != FN_ONE) {
      double s = 0.0;
#pragma unroll
      for (int a = 0; a < NV; ++a)
        s += mode == FN_P1 ? __ldg(w + v[a]) : __ldg(xw + 4 * size_t(v[a]) + comp);
      mean = s * (1.0 / NV);
    }
    acc = fma(meas, mean, acc);
  }
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int h = kFunctionalThreads / 2; h > 0; h >>= 1) {
    if (int(threadIdx.x) < h) red[threadIdx.x] += red[threadIdx.x + h];
    __syncthreads();
  }
  if (threadIdx.x == 0) partials[blockIdx.x] = red[0];
}

__global__ void __launch_bounds__(kFunctionalThreads) k_functional_sum(
    const double* __restrict__ partials, int n, double scale, double* __restrict__ out) {
  __shared__ double red[kFunctionalThreads];
  double acc = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) acc += partials[i];
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int h = kFunctionalThreads / 2; h > 0; h >>= 1) {
    if (int(threadIdx.x) < h) red[threadIdx.x] += red[threadIdx.x + h];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[0] = scale * red[0];
}

}  // namespace dev

namespace {

// Coefficient of a facet form: (P1 field?, scalar factor)
bool facet_coeff(const FormArgs& a, double& scale) {
  switch (a.f.coeff) {
    case DB2_COEFF_NONE: scale = 1.0; return false;
    case DB2_COEFF_CONSTANT: scale = a.f.constant[0]; return false;
    case DB2_COEFF_P1:
    case DB2_COEFF_P1_SCALED:
      if (!a.w) fail(DB2_ERR_ARGUMENT, "facet form coefficient is a P1 Function but no field was given");
      scale = a.f.coeff == DB2_COEFF_P1 ? 1.0 : a.f.constant[0];
      return true;
    default: fail(DB2_ERR_UNSUPPORTED, "coefficient kind %d is not provided for ds forms", a.f.coeff);
  }
}

dev::FacetParams facet_params(Pattern& P) {
  const FacetPlan& F = P.facet_plan();
  P.ensure_device();
  const Mesh& m = *P.V->mesh;
  dev::FacetParams p{};
  p.bnode = F.d_bnode.as<uint32_t>();
  p.binc_ptr = F.d_binc_ptr.as<uint32_t>();
  p.bverts = F.d_bverts.as<uint32_t>();
  p.bslot = F.d_bslot.as<uint8_t>();
  p.xw = m.d_x.as<double>();
  p.rowptr = P.d_rowptr.as<int32_t>();
  p.cols = P.d_cols.as<int32_t>();
  p.nnodes = P.V->nnodes;
  p.nverts = m.nv;
  // a partial row range (db2_pattern_set_row_range) takes the boundary nodes
  // inside it only: their facet rows are complete there, like the cell rows
  const int64_t r0 = P.row_begin, r1 = P.row_end < 0 ? P.V->nnodes : P.row_end;
  const auto lo = std::lower_bound(F.bnode.begin(), F.bnode.end(), uint32_t(r0));
  const auto hi = std::lower_bound(F.bnode.begin(), F.bnode.end(), uint32_t(r1));
  p.bn0 = int64_t(lo - F.bnode.begin());
  p.nbnodes = int64_t(hi - lo);
  p.bs = P.V->vsize;
  const OutputLayout o = output_layout(P);
  p.vbase = o.vbase;
  p.bstride = o.bstride;
  p.bbase = o.bbase;
  return p;
}

// Zero the pattern's rows inside its row range (all of them by default):
// CSR values of a scalar pattern, or the b entries (c, node) of every
// component c.
void zero_range_values(const Pattern& P, double* vals, cudaStream_t s) {
  const int64_t r0 = P.row_begin, r1 = P.row_end < 0 ? P.V->nnodes : P.row_end;
  const int64_t v0 = P.node_rowptr[r0], v1 = P.node_rowptr[r1];
  const OutputLayout o = output_layout(P);
  if (v1 > v0) cudaMemsetAsync(vals + v0 - o.vbase, 0, size_t(v1 - v0) * sizeof(double), s);
}
void zero_range_dofs(const Pattern& P, double* b, cudaStream_t s) {
  const int64_t r0 = P.row_begin, r1 = P.row_end < 0 ? P.V->nnodes : P.row_end;
  if (r1 <= r0) return;
  const OutputLayout o = output_layout(P);
  for (int c = 0; c < P.V->vsize; ++c)
    cudaMemsetAsync(b + int64_t(c) * o.bstride + r0 - o.bbase, 0, size_t(r1 - r0) * sizeof(double), s);
}

template <typename K>
void launch_rows(K kern, const dev::FacetParams& p, cudaStream_t s) {
  if (p.nbnodes == 0) return;
  kern<<<unsigned((p.nbnodes + 255) / 256), 256, 0, s>>>(p);
  count_launch();
}

}  // namespace

void launch_facet_vector(Pattern& P, const FormArgs& L, double* b, bool add_values,
                         const uint8_t* bc_flags, void* stream) {
  if (L.f.kind != DB2_FORM_FACET_LOAD) fail(DB2_ERR_ARGUMENT, "expected DB2_FORM_FACET_LOAD");
  const int D = P.V->mesh->tdim, deg = P.V->degree, bs = P.V->vsize;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  dev::FacetParams p = facet_params(P);
  double scale = 1.0;
  bool wp1 = facet_coeff(L, scale);
  if (bs != 1) {
    if (wp1) fail(DB2_ERR_UNSUPPORTED, "vector ds loads take a constant traction");
    for (int c = 0; c < 3; ++c) p.t[c] = L.f.coeff == DB2_COEFF_NONE ? 1.0 : L.f.constant[c];
  }
  p.scale = scale;
  p.w = L.w;
  p.b = b;
  p.bc_flags = bc_flags;
  if (!add_values) zero_range_dofs(P, b, s);
#define DB2_FV(D_, P_)                                                                   \
  if (D == D_ && deg == P_) {                                                            \
    if (wp1) launch_rows(dev::k_facet_vector<D_, P_, true>, p, s);                       \
    else launch_rows(dev::k_facet_vector<D_, P_, false>, p, s);                          \
  }
  DB2_FV(2, 1) DB2_FV(2, 2) DB2_FV(3, 1) DB2_FV(3, 2)
#undef DB2_FV
  check_cuda("facet vector launch");
}

void launch_facet_matrix(Pattern& P, const FormArgs& a, double* vals, bool add_values,
                         const uint8_t* bc_flags, const double* bc_vals, double* b, void* stream) {
  if (a.f.kind != DB2_FORM_FACET_MASS) fail(DB2_ERR_ARGUMENT, "expected DB2_FORM_FACET_MASS");
  if (P.V->vsize != 1) fail(DB2_ERR_UNSUPPORTED, "boundary mass on a vector space is not provided");
  if (bc_flags && (!bc_vals || !b)) fail(DB2_ERR_ARGUMENT, "Dirichlet data needs bc_vals and b");
  const int D = P.V->mesh->tdim, deg = P.V->degree;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  dev::FacetParams p = facet_params(P);
  double scale = 1.0;
  const bool wp1 = facet_coeff(a, scale);
  p.scale = scale;
  p.w = a.w;
  p.vals = vals;
  p.b = b;
  p.bc_flags = bc_flags;
  p.bc_vals = bc_vals;
  if (!add_values) zero_range_values(P, vals, s);
#define DB2_FM(D_, P_)                                                                   \
  if (D == D_ && deg == P_) {                                                            \
    if (wp1) launch_rows(dev::k_facet_matrix<D_, P_, true>, p, s);                       \
    else launch_rows(dev::k_facet_matrix<D_, P_, false>, p, s);                          \
  }
  DB2_FM(2, 1) DB2_FM(2, 2) DB2_FM(3, 1) DB2_FM(3, 2)
#undef DB2_FM
  check_cuda("facet matrix launch");
}

void launch_functional(Mesh& m, const FormArgs& M, double* out, void* stream) {
  const bool facet = M.f.kind == DB2_FORM_FACET_FUNCTIONAL;
  if (!facet && M.f.kind != DB2_FORM_FUNCTIONAL) fail(DB2_ERR_ARGUMENT, "not a functional");
  if (!out) fail(DB2_ERR_ARGUMENT, "out is NULL");
  const int D = m.tdim;
  if (D != 2 && D != 3) fail(DB2_ERR_UNSUPPORTED, "functionals on tdim %d", D);
  int mode = dev::FN_ONE, comp = 0;
  double scale = 1.0;
  switch (M.f.coeff) {
    case DB2_COEFF_NONE: break;
    case DB2_COEFF_CONSTANT: scale = M.f.constant[0]; break;
    case DB2_COEFF_P1:
    case DB2_COEFF_P1_SCALED:
      if (!M.w) fail(DB2_ERR_ARGUMENT, "functional coefficient is a P1 Function but no field was given");
      mode = dev::FN_P1;
      scale = M.f.coeff == DB2_COEFF_P1 ? 1.0 : M.f.constant[0];
      break;
    case DB2_COEFF_COORD:
      mode = dev::FN_COORD;
      scale = M.f.constant[0];
      comp = int(M.f.constant[1]);
      if (comp < 0 || comp >= D) fail(DB2_ERR_ARGUMENT, "coordinate component %d", comp);
      break;
    default: fail(DB2_ERR_ARGUMENT, "unknown coefficient kind %d", M.f.coeff);
  }
  m.ensure_device();
  int64_t n = m.nc;
  if (facet) {
    m.compute_exterior_facets();
    if (!m.d_ext_facets.ptr && !m.ext_facets.empty())
      m.d_ext_facets.upload(m.ext_facets.data(), m.ext_facets.size() * sizeof(uint32_t));
    n = int64_t(m.ext_facets.size());
  }
  if (!m.d_partials.ptr) m.d_partials.alloc(dev::kFunctionalBlocks * sizeof(double));
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  double* part = m.d_partials.as<double>();
  const double* xw = m.d_x.as<double>();
  const uint32_t* cells = m.d_cells.as<uint32_t>();
  const uint32_t* ext = m.d_ext_facets.as<uint32_t>();
#define DB2_FN(D_, F_)                                                                              \
  dev::k_functional<D_, F_><<<dev::kFunctionalBlocks, dev::kFunctionalThreads, 0, s>>>(             \
      xw, cells, ext, n, mode, M.w, comp, part)
  if (D == 2) {
    if (facet) DB2_FN(2, true);
    else DB2_FN(2, false);
  } else {
    if (facet) DB2_FN(3, true);
    else DB2_FN(3, false);
  }
#undef DB2_FN
  count_launch();
  dev::k_functional_sum<<<1, dev::kFunctionalThreads, 0, s>>>(part, dev::kFunctionalBlocks, scale,
                                                              out);
  count_launch();
  check_cuda("functional launch");
}

}  // namespace db2
