// action.cu -- matrix-free action y = A x (cell-wise element actions, then a
// per-row gather in cell order) and the adjoint (VJP) with respect to a P1
// coefficient.
#include <cuda_runtime.h>

#include <utility>

#include "launch.cuh"
#include "action_tc.cuh"

#include <algorithm>

namespace db2 {
namespace dev {

// Matrix-free action y = A x in two steps, without forming A.
//
// Step 1: the element action y_K = A_K x_K of every cell, by quadrature in
// barycentric coordinates (sum factorisation of the element kernels: the
// gradient of the trial function at a point, then its flux tested against
// every basis function), written once per (cell, component, local node).
// With lambda the barycentric coordinates and g_a = grad(lambda_a):
//   P2 basis derivatives  dphi_v/dl_a = delta_va (4 l_v - 1),
//                         dphi_(p,q)/dl_p = 4 l_q, dphi_(p,q)/dl_q = 4 l_p;
//   grad u = sum_a U_a g_a,  U_a = sum_j x_j dphi_j/dl_a;
//   y_j  += w |T| sum_a dphi_j/dl_a S_a,  S_a = flux . g_a,
// where the flux is kappa grad u (diffusion) or the stress row
// sigma_c = lambda div(u) e_c + mu (grad u + grad u^T)_c (elasticity; one
// thread per output component c).  The rules integrate the element
// integrands exactly: P1 -- the centroid (kappa linear, gradients
// constant); P2 diffusion -- degree 3 (kappa linear times two linear
// gradients); P2 elasticity -- degree 2.
template <int D, int DEG>
struct Quad;
template <int D>
struct Quad<D, 1> {  // centroid
  static constexpr int NQ = 1;
  __host__ __device__ static constexpr double w(int) { return 1.0; }
  __host__ __device__ static constexpr double lam(int, int) { return 1.0 / (D + 1); }
};
// Hammer-Marlowe-Stroud tetrahedron rule of degree 2: (a, b, b, b) and
// permutations, a = (5 + 3 sqrt 5) / 20, b = (5 - sqrt 5) / 20, weights 1/4.
template <>
struct Quad<3, 2> {
  static constexpr int NQ = 4;
  __host__ __device__ static constexpr double w(int) { return 0.25; }
  __host__ __device__ static constexpr double lam(int q, int a) {
    return a == q ? 0.5854101966249685 : 0.1381966011250105;
  }
};
// Stroud's degree-3 rules: tetrahedron -4/5 at the centroid and 9/20 at
// (1/2, 1/6, 1/6, 1/6) and permutations; triangle -27/48 at the centroid and
// 25/48 at (3/5, 1/5, 1/5) and permutations.
template <>
struct Quad<3, 3> {
  static constexpr int NQ = 5;
  __host__ __device__ static constexpr double w(int q) { return q == 0 ? -0.8 : 0.45; }
  __host__ __device__ static constexpr double lam(int q, int a) {
    return q == 0 ? 0.25 : (a == q - 1 ? 0.5 : 1.0 / 6.0);
  }
};
template <>
struct Quad<2, 3> {
  static constexpr int NQ = 4;
  __host__ __device__ static constexpr double w(int q) { return q == 0 ? -27.0 / 48.0 : 25.0 / 48.0; }
  __host__ __device__ static constexpr double lam(int q, int a) {
    return q == 0 ? 1.0 / 3.0 : (a == q - 1 ? 0.6 : 0.2);
  }
};

// grad(lambda_a) of the affine simplex and |T|.
template <int D>
__device__ __forceinline__ double bary_gradients(const double (&x)[D + 1][D], double (&g)[D + 1][D]) {
  Geometry<D> G;
  geometry(x, G);  // n[a] = det(J) grad(lambda_a), vol = |T|
  double det;
  if constexpr (D == 3) {
    det = (x[1][0] - x[0][0]) * G.n[1][0] + (x[1][1] - x[0][1]) * G.n[1][1] + (x[1][2] - x[0][2]) * G.n[1][2];
  } else {
    det = (x[1][0] - x[0][0]) * G.n[1][0] + (x[1][1] - x[0][1]) * G.n[1][1];
  }
  // 1/det from the geometry's 1/(D! |det|)
  const double inv = (D == 3 ? 6.0 : 2.0) * G.s * (det < 0.0 ? -1.0 : 1.0);
#pragma unroll
  for (int a = 0; a <= D; ++a)
#pragma unroll
    for (int r = 0; r < D; ++r) g[a][r] = G.n[a][r] * inv;
  return G.vol;
}

// U_a = sum_j x_j dphi_j/dl_a at barycentric point l, for one component.
template <int D, int P, typename CT>
__device__ __forceinline__ CT node_derivative(const CT (&xc)[El<D, P>::K], const double (&l)[D + 1], int a) {
  constexpr int NB = D + 1;
  if constexpr (P == 1) {
    return xc[a];
  } else {
    CT u = CT(4.0 * l[a] - 1.0) * xc[a];
#pragma unroll
    for (int e = 0; e < El<D, P>::NE; ++e) {
      const int p0 = edge_end(D, e, 0), p1 = edge_end(D, e, 1);
      if (p0 == a) u = fma(CT(4.0 * l[p1]), xc[NB + e], u);
      if (p1 == a) u = fma(CT(4.0 * l[p0]), xc[NB + e], u);
    }
    return u;
  }
}

// y_j += sum_a dphi_j/dl_a S_a at barycentric point l.
template <int D, int P, typename CT>
__device__ __forceinline__ void test_basis(const CT (&S)[D + 1], const double (&l)[D + 1],
                                           double (&y)[El<D, P>::K]) {
  constexpr int NB = D + 1;
#pragma unroll
  for (int v = 0; v < NB; ++v) y[v] += double(P == 1 ? S[v] : CT(4.0 * l[v] - 1.0) * S[v]);
  if constexpr (P == 2) {
#pragma unroll
    for (int e = 0; e < El<D, P>::NE; ++e) {
      const int p0 = edge_end(D, e, 0), p1 = edge_end(D, e, 1);
      y[NB + e] += double(fma(CT(4.0 * l[p1]), S[p0], CT(4.0 * l[p0]) * S[p1]));
    }
  }
}

// Block size and register cap of step 1.  Residency is set per SM
// sub-partition (16,384 registers: 5 warps at 81-96 registers per thread,
// 6 at up to 80) and in whole blocks.
#ifndef DB2_APPLY_THREADS
#define DB2_APPLY_THREADS 128
#endif
#ifndef DB2_APPLY_MAXNREG_P2DIFF
#define DB2_APPLY_MAXNREG_P2DIFF 80
#endif
#ifndef DB2_APPLY_MAXNREG_ELAS
#define DB2_APPLY_MAXNREG_ELAS 128
#endif
template <int P, int FORM>
constexpr int apply_maxnreg() {
  return FORM == FORM_ELAS ? DB2_APPLY_MAXNREG_ELAS : P == 2 ? DB2_APPLY_MAXNREG_P2DIFF : 255;
}
template <int D, int P, int FORM, bool KP1, typename CT>
__global__ void __maxnreg__((apply_maxnreg<P, FORM>())) k_apply_cells(const AsmParams p, int64_t ncells,
                                                     const double* __restrict__ xin,
                                                     CT* __restrict__ ycell) {
  constexpr int NB = D + 1, K = El<D, P>::K;
  constexpr bool ELAS = FORM == FORM_ELAS;
  constexpr int BS = ELAS ? D : 1;
  using Q = Quad<D, P == 1 ? 1 : (ELAS ? 2 : 3)>;
  const int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  const int64_t cell = ELAS ? t / D : t;
  const int c = ELAS ? int(t - cell * D) : 0;
  if (cell >= ncells) return;
  double xv[NB][D], kap[NB];
  uint32_t vid[NB];
#pragma unroll
  for (int a = 0; a < NB; ++a) {
    double f;
    vid[a] = __ldg(p.cells + size_t(cell) * NB + a);
    load_vertex<D, false>(p, vid[a], xv[a], kap[a], f);
  }
  double g[NB][D];
  const double vol = bary_gradients<D>(xv, g);
  CT gc[NB][D];
#pragma unroll
  for (int a = 0; a < NB; ++a)
#pragma unroll
    for (int r = 0; r < D; ++r) gc[a][r] = CT(g[a][r]);
  CT xc[BS][K];
#pragma unroll
  for (int j = 0; j < K; ++j) {
    // vertex nodes are numbered as the vertices (natural numbering)
    const uint32_t node = j < NB ? vid[j] : __ldg(p.cell_nodes + size_t(cell) * K + j);
#pragma unroll
    for (int e = 0; e < BS; ++e) xc[e][j] = CT(__ldg(xin + int64_t(e) * p.nnodes + node));
  }
  double y[K];
#pragma unroll
  for (int j = 0; j < K; ++j) y[j] = 0.0;
#pragma unroll
  for (int q = 0; q < Q::NQ; ++q) {
    double l[NB];
#pragma unroll
    for (int a = 0; a < NB; ++a) l[a] = Q::lam(q, a);
    double wq = Q::w(q) * vol;
    // grad u: gu[e][d] = sum_a U_a^e g_a[d]
    CT gu[BS][D];
#pragma unroll
    for (int e = 0; e < BS; ++e) {
#pragma unroll
      for (int d = 0; d < D; ++d) gu[e][d] = CT(0);
#pragma unroll
      for (int a = 0; a < NB; ++a) {
        const CT u = node_derivative<D, P, CT>(xc[e], l, a);
#pragma unroll
        for (int d = 0; d < D; ++d) gu[e][d] = fma(u, gc[a][d], gu[e][d]);
      }
    }
    CT flux[D];
    if constexpr (ELAS) {
      CT div = gu[0][0];
#pragma unroll
      for (int d = 1; d < D; ++d) div += gu[d][d];
#pragma unroll
      for (int d = 0; d < D; ++d) flux[d] = CT(p.mu) * (gu[c][d] + gu[d][c]);
      flux[c] = fma(CT(p.lmbda), div, flux[c]);
    } else {
      double k = p.kscale;
      if constexpr (KP1) {
        double kq = 0.0;
#pragma unroll
        for (int a = 0; a < NB; ++a) kq = fma(kap[a], l[a], kq);
        k *= kq;
      }
#pragma unroll
      for (int d = 0; d < D; ++d) flux[d] = CT(k) * gu[0][d];
    }
    CT S[NB];
#pragma unroll
    for (int a = 0; a < NB; ++a) {
      CT sa = flux[0] * gc[a][0];
#pragma unroll
      for (int d = 1; d < D; ++d) sa = fma(flux[d], gc[a][d], sa);
      S[a] = CT(wq) * sa;
    }
    test_basis<D, P, CT>(S, l, y);
  }
  if constexpr (ELAS) {
    // cell-major (cell, j, c): a node's three components of one cell are
    // adjacent, and the cell's three component threads fill one block
#pragma unroll
    for (int j = 0; j < K; ++j) ycell[(size_t(cell) * K + j) * BS + c] = y[j];
  } else {
    // each value goes to its incidence slot (node-contiguous, ascending cell
    // order), so that step 2 reads every row's terms contiguously
#pragma unroll
    for (int j = 0; j < K; ++j) ycell[__ldg(p.cell_inc + size_t(cell) * K + j)] = y[j];
  }
}

// Step 2: y = sum of the element actions of the node's incident cells, in
// ascending cell order -- a fixed order, so the result is bitwise
// repeatable.  Scalar forms (one thread per row) read the terms
// contiguously (incidence order).  Elasticity (one thread per node, all
// components) finds them through the incidence words (cell | local node <<
// 28) in the cell-major array, the three components of a term adjacent --
// measured faster than component planes in incidence order for its three
// component threads per cell (0.33 ms against 0.46 ms per action, vector P2
// on UnitCubeMesh(48)).
template <int BS, int K, bool INC, typename ST = double>
__global__ void __launch_bounds__(256) k_apply_gather(const uint32_t* __restrict__ inc_ptr,
                                                      const uint32_t* __restrict__ inc,
                                                      int64_t nnodes, const ST* __restrict__ ycell,
                                                      double* __restrict__ y) {
  const int64_t node = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (node >= nnodes) return;
  const uint32_t s0 = __ldg(inc_ptr + node), s1 = __ldg(inc_ptr + node + 1);
  double acc[BS];
#pragma unroll
  for (int c = 0; c < BS; ++c) acc[c] = 0.0;
  if constexpr (INC) {
    for (uint32_t s = s0; s < s1; ++s) acc[0] += double(__ldg(ycell + s));
  } else {
    for (uint32_t s = s0; s < s1; ++s) {
      const uint32_t w = __ldg(inc + s);
      const ST* t = ycell + (size_t(w & 0x0fffffffu) * K + (w >> 28)) * BS;
#pragma unroll
      for (int c = 0; c < BS; ++c) acc[c] += double(__ldg(t + c));
    }
  }
#pragma unroll
  for (int c = 0; c < BS; ++c) y[int64_t(c) * nnodes + node] = acc[c];
}

// Adjoint, step 1, the part of local node LI of the cell (a compile-time
// relabelling, so the permuted geometry tensor is register renaming):
// acc[a] += sum_j gA_(LI,j) dA^K_(LI,j)/dkappa_a + gb_LI db^K_LI/dkappa_a.
// Wn[a][b] = n_a . n_b in the cell's own vertex order; under the relabelling
// n'_a = +-n_perm[a], so W'_ab = Wn[perm[a]][perm[b]] (|det J| unchanged).
template <int D, int P, bool LOADK, typename CT, int LI>
__device__ __forceinline__ void vjp_node(const AsmParams& p, int64_t cell,
                                         const double (&Wn)[D + 1][D + 1], double s, double vol,
                                         const double (&fv)[D + 1], const double* __restrict__ gA,
                                         const double* __restrict__ gb, double (&acc)[D + 1]) {
  using E = El<D, P>;
  using R = Rows<D, P, CT>;
  constexpr int NB = D + 1;
  constexpr uint32_t code = perm_code(D, LI);
  constexpr bool vertex = LI <= D;
  const uint32_t ii = __ldg(p.cell_inc + size_t(cell) * E::K + LI);
  const uint32_t node = __ldg(p.cell_nodes + size_t(cell) * E::K + LI);
  const double* grow = gA + __ldg(p.node_rowptr + node);
  // gA at the row's slots, in the relabelled local order
  double g[E::K];
  const Rec<D, P> rr = load_rec<D, P>(p, rec_index<D, P>(p, node, ii - __ldg(p.inc_ptr + node)));
#pragma unroll
  for (int j = 0; j < E::K; ++j) g[j] = __ldg(grow + rr.slot(j));
  auto pm = [](int a) { return int((code >> (2 * a)) & 3u); };
  CT W0[1][NB];
  CT W1[2][NB];
  // W times the generated rows' scale (see element_rows.h)
  const double sv = s * (p.kscale * R::sv_kp1);
#pragma unroll
  for (int b = 0; b < NB; ++b) W0[0][b] = CT(Wn[pm(0)][pm(b)] * sv);
  if constexpr (P == 2) {
    const double se = s * (p.kscale * R::se_kp1);
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
      for (int b = 0; b < NB; ++b) W1[a][b] = CT(Wn[pm(a)][pm(b)] * se);
  }
  CT lk[NB];
  if constexpr (LOADK) {
    CT fc[NB];
#pragma unroll
    for (int a = 0; a < NB; ++a) fc[a] = CT(fv[pm(a)]);
    if constexpr (P == 2 && !vertex) R::e_kfp1(fc, lk);
    else R::v_kfp1(fc, lk);
  }
  const double gbi = LOADK ? __ldg(gb + node) : 0.0;
#pragma unroll
  for (int m = 0; m < NB; ++m) {
    CT unit[NB];
#pragma unroll
    for (int a = 0; a < NB; ++a) unit[a] = CT(a == m ? 1 : 0);
    CT d[E::K];
    if constexpr (P == 1 || vertex) R::v_kp1(W0, unit, d);
    else R::e_kp1(W1, unit, d);
    double t = 0.0;
#pragma unroll
    for (int j = 0; j < E::K; ++j) t = fma(g[j], double(d[j]), t);
    if constexpr (LOADK) t = fma(gbi, vol * double(lk[m]) * p.fc[0], t);
    // relabelled vertex m is original local vertex perm[m]
    acc[pm(m)] += t;
  }
}

template <int D, int P, bool LOADK, typename CT, int... LI>
__device__ __forceinline__ void vjp_nodes(const AsmParams& p, int64_t cell,
                                          const double (&Wn)[D + 1][D + 1], double s, double vol,
                                          const double (&fv)[D + 1], const double* gA,
                                          const double* gb, double (&acc)[D + 1],
                                          std::integer_sequence<int, LI...>) {
  (vjp_node<D, P, LOADK, CT, LI>(p, cell, Wn, s, vol, fv, gA, gb, acc), ...);
}

// Adjoint, step 1 (one thread per cell): t[cell][m] = sum_{i,j in cell}
// gA_ij dA^K_ij/dkappa_m + sum_i gb_i db^K_i/dkappa_m for the P1 kappa
// basis functions m of the cell.  The cell's vertices and geometry are
// loaded and computed once; each local node's relabelled geometry tensor is
// a permutation of the cell's.
// Register caps: the P2 node parts (ten of them, inlined) would take up to
// 174 registers uncapped; P1 cells need no more than 64.
template <int P>
constexpr int vjp_maxnreg() {
  return P == 1 ? 64 : 128;
}
template <int D, int P, bool LOADK, typename CT>
__global__ void __maxnreg__((vjp_maxnreg<P>())) k_vjp_cells(const AsmParams p, int64_t ncells,
                                                   const double* __restrict__ gA,
                                                   const double* __restrict__ gb,
                                                   double* __restrict__ t) {
  using E = El<D, P>;
  constexpr int NB = D + 1;
  const int64_t cell = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (cell >= ncells) return;
  uint32_t v[NB];
  load_verts<D>(p, uint32_t(cell), v);
  double x[NB][D], kap_unused[NB], f_unused[NB];
  load_vertex_data<D, false>(p, v, x, kap_unused, f_unused);
  double fv[NB];
#pragma unroll
  for (int a = 0; a < NB; ++a) fv[a] = LOADK ? __ldg(p.f + v[a]) : 0.0;
  Geometry<D> G;
  geometry(x, G);
  double Wn[NB][NB];
#pragma unroll
  for (int a = 0; a < NB; ++a)
#pragma unroll
    for (int b = a; b < NB; ++b) Wn[a][b] = Wn[b][a] = ndot<D>(G, a, b);
  double acc[NB];
#pragma unroll
  for (int a = 0; a < NB; ++a) acc[a] = 0.0;
  vjp_nodes<D, P, LOADK, CT>(p, cell, Wn, G.s, G.vol, fv, gA, gb, acc,
                             std::make_integer_sequence<int, E::K>{});
  // in vertex-incidence order (vertex nodes come first in the node-contiguous
  // incidence array), so that step 2 reads each vertex's terms contiguously
  for (int a = 0; a < NB; ++a) t[__ldg(p.cell_inc + size_t(cell) * E::K + a)] = acc[a];
}

// Adjoint, step 2 (one thread per vertex): dkappa[v] = sum over cells around
// v, in cell order, of their terms for v (contiguous: incidence order).
template <int D, int P>
__global__ void __launch_bounds__(256) k_vjp_vertices(const AsmParams p, int64_t nv,
                                                      const double* __restrict__ t,
                                                      double* __restrict__ dk) {
  const int64_t v = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (v >= nv) return;
  double s = 0.0;
  const uint32_t s1 = __ldg(p.inc_ptr + v + 1);
  for (uint32_t ii = __ldg(p.inc_ptr + v); ii < s1; ++ii) s += __ldg(t + ii);
  dk[v] = s;
}

template <int D, int P, int FORM, bool KP1, typename CT>
void run_apply(const Pattern& Pt, const AsmParams& p, const double* x, double* y, cudaStream_t s) {
  constexpr int K = El<D, P>::K, BS = FORM == FORM_ELAS ? D : 1, n = BS * K;
  const int64_t nc = Pt.V->mesh->nc;
  // element actions in the contraction type (the FP32 path moves half the
  // bytes); the ordered gather sums them in FP64
  const size_t need = size_t(nc) * n * sizeof(CT);
  if (Pt.d_cellvals.bytes < need) Pt.d_cellvals.alloc(need);
  CT* ycell = Pt.d_cellvals.as<CT>();
  const int64_t threads = nc * (FORM == FORM_ELAS ? D : 1);
  if (threads > 0) {
    constexpr int bt = DB2_APPLY_THREADS;
    k_apply_cells<D, P, FORM, KP1, CT><<<unsigned((threads + bt - 1) / bt), bt, 0, s>>>(p, nc, x, ycell);
    count_launch();
    check_cuda("apply launch");
  }
  k_apply_gather<BS, K, FORM != FORM_ELAS, CT><<<unsigned((p.nnodes + 255) / 256), 256, 0, s>>>(
      p.inc_ptr, p.inc, p.nnodes, ycell, y);
  count_launch();
  check_cuda("apply gather launch");
}

// The FP32-contraction action of P2 diffusion on tetrahedra: element actions
// by the tensor-core kernel (action_tc.cuh), then the same ordered gather.
template <bool KP1>
void run_apply_tc(const Pattern& Pt, const AsmParams& p, const double* x, double* y, cudaStream_t s) {
  const int64_t nc = Pt.V->mesh->nc;
  const size_t need = size_t(nc) * 10 * sizeof(float);
  if (Pt.d_cellvals.bytes < need) Pt.d_cellvals.alloc(need);
  float* ycell = Pt.d_cellvals.as<float>();
  if (nc > 0) {
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    // persistent: the 5 CTAs per SM the launch bounds provide for (registers
    // <= 102; 5 x 30 KB of shared memory; 5 x 64 of the 512 tensor-memory
    // columns)
    const int64_t ntiles = (nc + kTcM - 1) / kTcM;
    const unsigned grid = unsigned(std::min<int64_t>(ntiles, int64_t(sms) * 5));
    k_apply_tc_p2<KP1><<<grid, kTcM, sizeof(TcSmem), s>>>(p, nc, x, ycell);
    count_launch();
    check_cuda("tensor-core apply launch");
  }
  k_apply_gather<1, 10, true, float><<<unsigned((p.nnodes + 255) / 256), 256, 0, s>>>(p.inc_ptr, p.inc,
                                                                                     p.nnodes, ycell, y);
  count_launch();
  check_cuda("apply gather launch");
}

}  // namespace dev

int tensor_core_status() {
  int v = 0;
  const cudaError_t e = cudaMemcpyFromSymbol(&v, dev::g_tc_status, sizeof(int));
  if (e != cudaSuccess) fail(DB2_ERR_CUDA, "reading the tensor-core status: %s", cudaGetErrorString(e));
  return v;
}

dev::AsmParams make_params(const Pattern& P);
void pack_vertex_records(const Pattern& P, const double* kappa, const double* f, void* stream);

void launch_apply(const Pattern& P, const FormArgs& a, int precision, const double* x, double* y,
                  void* stream) {
  dev::AsmParams p = make_params(P);
  const int D = P.V->mesh->tdim, deg = P.V->degree;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const bool tc = precision == DB2_FP32_TENSOR_CORE;
  const bool fp32 = precision == DB2_FP32_CONTRACT || tc;
  if (precision != DB2_FP64 && !fp32) fail(DB2_ERR_ARGUMENT, "unknown precision %d", precision);
  bool kp1 = false;
  if (a.f.kind == DB2_FORM_DIFFUSION) {
    if (P.bs != 1) fail(DB2_ERR_UNSUPPORTED, "diffusion form on a vector space");
    p.kscale = a.f.coeff == DB2_COEFF_CONSTANT || a.f.coeff == DB2_COEFF_P1_SCALED ? a.f.constant[0] : 1.0;
    kp1 = a.f.coeff == DB2_COEFF_P1 || a.f.coeff == DB2_COEFF_P1_SCALED;
    if (kp1 && !a.w) fail(DB2_ERR_ARGUMENT, "P1 coefficient field missing");
    p.kappa = a.w;
    pack_vertex_records(P, kp1 ? a.w : nullptr, nullptr, stream);
    if (tc) {
      if (D != 3 || deg != 2)
        fail(DB2_ERR_UNSUPPORTED, "the tensor-core action is for P2 tetrahedra");
      // FP32 contraction on the tensor cores
      if (kp1) dev::run_apply_tc<true>(P, p, x, y, s);
      else dev::run_apply_tc<false>(P, p, x, y, s);
      return;
    }
#define DB2_AP(D_, P_)                                                                  \
  if (D == D_ && deg == P_) {                                                           \
    if (kp1) {                                                                          \
      if (fp32) dev::run_apply<D_, P_, dev::FORM_DIFF, true, float>(P, p, x, y, s);     \
      else dev::run_apply<D_, P_, dev::FORM_DIFF, true, double>(P, p, x, y, s);         \
    } else {                                                                            \
      if (fp32) dev::run_apply<D_, P_, dev::FORM_DIFF, false, float>(P, p, x, y, s);    \
      else dev::run_apply<D_, P_, dev::FORM_DIFF, false, double>(P, p, x, y, s);        \
    }                                                                                   \
    return;                                                                             \
  }
    DB2_AP(3, 1) DB2_AP(3, 2) DB2_AP(2, 1) DB2_AP(2, 2)
#undef DB2_AP
  } else if (a.f.kind == DB2_FORM_ELASTICITY) {
    if (D != 3 || P.bs != 3) fail(DB2_ERR_UNSUPPORTED, "elasticity needs a 3D vector space");
    if (tc) fail(DB2_ERR_UNSUPPORTED, "the tensor-core action is for P2 diffusion");
    p.mu = a.f.mu;
    p.lmbda = a.f.lmbda;
    if (deg == 1) {
      if (fp32) dev::run_apply<3, 1, dev::FORM_ELAS, false, float>(P, p, x, y, s);
      else dev::run_apply<3, 1, dev::FORM_ELAS, false, double>(P, p, x, y, s);
    } else {
      if (fp32) dev::run_apply<3, 2, dev::FORM_ELAS, false, float>(P, p, x, y, s);
      else dev::run_apply<3, 2, dev::FORM_ELAS, false, double>(P, p, x, y, s);
    }
    return;
  }
  fail(DB2_ERR_UNSUPPORTED, "matrix-free action not provided for this form/element");
}

void preload_vjp_kernels() {
  cudaFuncAttributes at;
  cudaError_t e = cudaSuccess;
  auto get = [&](const void* f) {
    const cudaError_t r = cudaFuncGetAttributes(&at, f);
    if (r != cudaSuccess) e = r;
  };
#define DB2_VJP_LOAD(D_, P_)                                                  \
  get((const void*)dev::k_vjp_cells<D_, P_, true, float>);                    \
  get((const void*)dev::k_vjp_cells<D_, P_, true, double>);                   \
  get((const void*)dev::k_vjp_cells<D_, P_, false, float>);                   \
  get((const void*)dev::k_vjp_cells<D_, P_, false, double>);                  \
  get((const void*)dev::k_vjp_vertices<D_, P_>);
  DB2_VJP_LOAD(3, 1) DB2_VJP_LOAD(3, 2) DB2_VJP_LOAD(2, 1) DB2_VJP_LOAD(2, 2)
#undef DB2_VJP_LOAD
  if (e != cudaSuccess) fail(DB2_ERR_CUDA, "loading the adjoint kernels: %s", cudaGetErrorString(e));
}

size_t vjp_scratch_doubles(const Pattern& P) {
  return size_t(P.V->mesh->nc) * (P.V->mesh->tdim + 1);
}

void launch_vjp(const Pattern& P, const FormArgs& a, const FormArgs& L, int precision,
                const double* gA, const double* gb, double* dkappa, double* scratch,
                void* stream) {
  if (a.f.kind != DB2_FORM_DIFFUSION || P.bs != 1)
    fail(DB2_ERR_UNSUPPORTED, "the adjoint is provided for kappa*grad(u).grad(v)*dx on scalar spaces");
  if (!(a.f.coeff == DB2_COEFF_P1 || a.f.coeff == DB2_COEFF_P1_SCALED))
    fail(DB2_ERR_ARGUMENT, "the adjoint is with respect to a P1 kappa");
  const bool tc = precision == DB2_FP32_TENSOR_CORE;
  const bool fp32 = precision == DB2_FP32_CONTRACT || tc;
  if (precision != DB2_FP64 && !fp32) fail(DB2_ERR_ARGUMENT, "unknown precision %d", precision);
  dev::AsmParams p = make_params(P);
  p.kscale = a.f.coeff == DB2_COEFF_P1_SCALED ? a.f.constant[0] : 1.0;
  p.kappa = a.w;
  // L = kappa * f * v * dx contributes when its coefficient is P1_SCALED
  // (the kappa-weighted load); any other load does not depend on kappa.
  const bool loadk = gb && L.f.kind == DB2_FORM_LOAD &&
                     (L.f.coeff == DB2_COEFF_P1_SCALED || L.f.coeff == DB2_COEFF_P1_KAPPA);
  if (loadk) {
    if (!L.w) fail(DB2_ERR_ARGUMENT, "kappa-weighted load needs its P1 field f");
    p.f = L.w;
    p.fc[0] = L.f.coeff == DB2_COEFF_P1_KAPPA ? L.f.constant[0] : 1.0;
  }
  const int D = P.V->mesh->tdim, deg = P.V->degree;
  const int64_t nc = P.V->mesh->nc, nv = P.V->mesh->nv;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const unsigned bc = unsigned((nc + 255) / 256), bv = unsigned((nv + 255) / 256);
#define DB2_VJP(D_, P_)                                                                        \
  if (D == D_ && deg == P_) {                                                                  \
    if (loadk) {                                                                               \
      if (fp32) dev::k_vjp_cells<D_, P_, true, float><<<bc, 256, 0, s>>>(p, nc, gA, gb, scratch); \
      else dev::k_vjp_cells<D_, P_, true, double><<<bc, 256, 0, s>>>(p, nc, gA, gb, scratch);  \
    } else {                                                                                   \
      if (fp32) dev::k_vjp_cells<D_, P_, false, float><<<bc, 256, 0, s>>>(p, nc, gA, gb, scratch); \
      else dev::k_vjp_cells<D_, P_, false, double><<<bc, 256, 0, s>>>(p, nc, gA, gb, scratch); \
    }                                                                                          \
    dev::k_vjp_vertices<D_, P_><<<bv, 256, 0, s>>>(p, nv, scratch, dkappa);                         \
    count_launch(2);                                                                           \
    check_cuda("vjp launch");                                                                  \
    return;                                                                                    \
  }
  DB2_VJP(3, 1) DB2_VJP(3, 2) DB2_VJP(2, 1) DB2_VJP(2, 2)
#undef DB2_VJP
  fail(DB2_ERR_UNSUPPORTED, "adjoint not provided for this element");
}

}  // namespace db2
