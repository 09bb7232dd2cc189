// action.cu -- matrix-free action y = A x and the adjoint (VJP) with respect
// to a P1 coefficient, on the same row-gather plan as assembly.
#include <cuda_runtime.h>

#include "launch.cuh"

namespace db2 {
namespace dev {

// y[(c,i)] = sum over cells K around node i of sum_{e,j} A^K_{(c,i),(e,j)} x[(e,j)]
// (one thread per dof row, register accumulation in cell order; the x index
// of column slot q of block e is the CSR column itself).
template <int D, int P, int FORM, bool KP1, typename CT>
__global__ void __launch_bounds__(256) k_apply(const AsmParams p, const double* __restrict__ xin,
                                               double* __restrict__ y) {
  using E = El<D, P>;
  constexpr int BS = FORM == FORM_ELAS ? D : 1;
  const int64_t r = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (r >= p.nnodes * BS) return;
  const int c = int(r / p.nnodes);
  const uint32_t node = uint32_t(r - int64_t(c) * p.nnodes);
  const int32_t ra = __ldg(p.node_rowptr + node);
  const int32_t L = __ldg(p.node_rowptr + node + 1) - ra;
  const int32_t* crow = p.cols + int64_t(c) * BS * p.nnz_node + int64_t(BS) * ra;
  const uint32_t cnt = __ldg(p.inc_ptr + node + 1) - __ldg(p.inc_ptr + node);
  const uint32_t rbase = __ldg(p.rec_goff + (node >> 5)) + (node & 31u);
  const RowFix<D> F = load_row_fix<D, P, false>(p, node);
  double acc = 0.0;
  for (uint32_t m = 0; m < cnt; ++m) {
    const Rec<D, P> rr = load_rec<D, P>(p, rbase + 32u * m);
    double x[D + 1][D], kap[D + 1], fv[D + 1];
    record_cell<D, P, false>(p, F, rr, x, kap, fv);
    Geometry<D> G;
    geometry(x, G);
#pragma unroll 1
    for (int e = 0; e < BS; ++e) {
      CT out[E::K];
      element_row<D, P, FORM, KP1, CT>(p, G, F.nfix == 1, c, e, kap, out);
#pragma unroll
      for (int j = 0; j < E::K; ++j)
        acc = fma(double(out[j]), __ldg(xin + __ldg(crow + e * L + rr.slot(j))), acc);
    }
  }
  y[r] = acc;
}

// Adjoint, step 1 (one thread per cell): t[cell][m] = sum_{i,j in cell}
// gA_ij dA^K_ij/dkappa_m + sum_i gb_i db^K_i/dkappa_m for the P1 kappa
// basis functions m of the cell.
template <int D, int P, bool LOADK, typename CT>
__global__ void __launch_bounds__(256) k_vjp_cells(const AsmParams p, int64_t ncells,
                                                   const double* __restrict__ gA,
                                                   const double* __restrict__ gb,
                                                   double* __restrict__ t) {
  using E = El<D, P>;
  using R = Rows<D, P, CT>;
  constexpr int NB = D + 1;
  const int64_t cell = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (cell >= ncells) return;
  double acc[NB];
  for (int a = 0; a < NB; ++a) acc[a] = 0.0;
  const uint32_t* cn = p.cell_nodes + size_t(cell) * E::K;
  for (int li = 0; li < E::K; ++li) {
    const uint32_t ii = __ldg(p.cell_inc + size_t(cell) * E::K + li);
    const uint32_t node = __ldg(cn + li);
    const double* grow = gA + __ldg(p.node_rowptr + node);
    const uint32_t code = perm_of<D>(li);
    uint32_t v[D + 1], pv[D + 1];
    load_verts<D>(p, uint32_t(cell), v);
    relabel<D>(v, code, pv);
    double x[D + 1][D], kap_unused[D + 1], f_unused[D + 1];
    load_vertex_data<D, false>(p, pv, x, kap_unused, f_unused);
    Geometry<D> G;
    geometry(x, G);
    const bool vertex = li <= D;
    // gA at the row's slots, in the relabelled local order
    double g[E::K];
    const Rec<D, P> rr = load_rec<D, P>(p, rec_index<D, P>(p, node, ii - __ldg(p.inc_ptr + node)));
#pragma unroll
    for (int j = 0; j < E::K; ++j) g[j] = __ldg(grow + rr.slot(j));
    CT W0[1][NB];
    CT W1[2][NB];
    // W times the generated rows' scale (see element_rows.h)
    for (int b = 0; b < NB; ++b) W0[0][b] = CT(ndot<D>(G, 0, b) * (G.s * (p.kscale * R::sv_kp1)));
    if constexpr (P == 2)
      for (int a = 0; a < 2; ++a)
        for (int b = 0; b < NB; ++b)
          W1[a][b] = CT(ndot<D>(G, a, b) * (G.s * (p.kscale * R::se_kp1)));
    double fv[NB];
    if constexpr (LOADK)
      for (int a = 0; a < NB; ++a) fv[a] = __ldg(p.f + pv[a]);
    CT lk[NB];
    if constexpr (LOADK) {
      CT fc[NB];
      for (int a = 0; a < NB; ++a) fc[a] = CT(fv[a]);
      if constexpr (P == 2) {
        if (vertex) R::v_kfp1(fc, lk);
        else R::e_kfp1(fc, lk);
      } else {
        R::v_kfp1(fc, lk);
      }
    }
    const double gbi = LOADK ? __ldg(gb + node) : 0.0;
    for (int m = 0; m < NB; ++m) {
      CT unit[NB];
      for (int a = 0; a < NB; ++a) unit[a] = CT(a == m ? 1 : 0);
      CT d[E::K];
      if (P == 1 || vertex) R::v_kp1(W0, unit, d);
      else if constexpr (P == 2) R::e_kp1(W1, unit, d);
      double s = 0.0;
      for (int j = 0; j < E::K; ++j) s = fma(g[j], double(d[j]), s);
      if constexpr (LOADK) s = fma(gbi, G.vol * double(lk[m]) * p.fc[0], s);
      // relabelled vertex m is original local vertex perm[m]
      const int orig = int((code >> (2 * m)) & 3u);
      for (int a = 0; a < NB; ++a)
        if (a == orig) acc[a] += s;
    }
  }
  for (int a = 0; a < NB; ++a) t[cell * NB + a] = acc[a];
}

// Adjoint, step 2 (one thread per vertex): dkappa[v] = sum over cells around
// v, in cell order, of t[cell][local index of v].
template <int D, int P>
__global__ void __launch_bounds__(256) k_vjp_vertices(const AsmParams p, int64_t nv,
                                                      const double* __restrict__ t,
                                                      double* __restrict__ dk) {
  const int64_t v = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (v >= nv) return;
  double s = 0.0;
  for (uint32_t ii = __ldg(p.inc_ptr + v); ii < __ldg(p.inc_ptr + v + 1); ++ii) {
    const uint32_t word = __ldg(p.inc + ii);
    s += __ldg(t + size_t(word & 0x0fffffffu) * (D + 1) + (word >> 28));
  }
  dk[v] = s;
}

template <int D, int P, int FORM, bool KP1, typename CT>
void run_apply(const AsmParams& p, int bs, const double* x, double* y, cudaStream_t s) {
  const int64_t n = p.nnodes * bs;
  k_apply<D, P, FORM, KP1, CT><<<unsigned((n + 255) / 256), 256, 0, s>>>(p, x, y);
  count_launch();
  check_cuda("apply launch");
}

}  // namespace dev

dev::AsmParams make_params(const Pattern& P);
void pack_vertex_records(const Pattern& P, const double* kappa, const double* f, void* stream);

void launch_apply(const Pattern& P, const FormArgs& a, int precision, const double* x, double* y,
                  void* stream) {
  dev::AsmParams p = make_params(P);
  const int D = P.V->mesh->tdim, deg = P.V->degree;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const bool fp32 = precision == DB2_FP32_CONTRACT;
  if (precision != DB2_FP64 && !fp32) fail(DB2_ERR_ARGUMENT, "unknown precision %d", precision);
  bool kp1 = false;
  if (a.f.kind == DB2_FORM_DIFFUSION) {
    if (P.bs != 1) fail(DB2_ERR_UNSUPPORTED, "diffusion form on a vector space");
    p.kscale = a.f.coeff == DB2_COEFF_CONSTANT || a.f.coeff == DB2_COEFF_P1_SCALED ? a.f.constant[0] : 1.0;
    kp1 = a.f.coeff == DB2_COEFF_P1 || a.f.coeff == DB2_COEFF_P1_SCALED;
    if (kp1 && !a.w) fail(DB2_ERR_ARGUMENT, "P1 coefficient field missing");
    p.kappa = a.w;
    pack_vertex_records(P, kp1 ? a.w : nullptr, nullptr, stream);
#define DB2_AP(D_, P_)                                                                  \
  if (D == D_ && deg == P_) {                                                           \
    if (kp1) {                                                                          \
      if (fp32) dev::run_apply<D_, P_, dev::FORM_DIFF, true, float>(p, 1, x, y, s);     \
      else dev::run_apply<D_, P_, dev::FORM_DIFF, true, double>(p, 1, x, y, s);         \
    } else {                                                                            \
      if (fp32) dev::run_apply<D_, P_, dev::FORM_DIFF, false, float>(p, 1, x, y, s);    \
      else dev::run_apply<D_, P_, dev::FORM_DIFF, false, double>(p, 1, x, y, s);        \
    }                                                                                   \
    return;                                                                             \
  }
    DB2_AP(3, 1) DB2_AP(3, 2) DB2_AP(2, 1) DB2_AP(2, 2)
#undef DB2_AP
  } else if (a.f.kind == DB2_FORM_ELASTICITY) {
    if (D != 3 || P.bs != 3) fail(DB2_ERR_UNSUPPORTED, "elasticity needs a 3D vector space");
    p.mu = a.f.mu;
    p.lmbda = a.f.lmbda;
    if (deg == 1) {
      if (fp32) dev::run_apply<3, 1, dev::FORM_ELAS, false, float>(p, 3, x, y, s);
      else dev::run_apply<3, 1, dev::FORM_ELAS, false, double>(p, 3, x, y, s);
    } else {
      if (fp32) dev::run_apply<3, 2, dev::FORM_ELAS, false, float>(p, 3, x, y, s);
      else dev::run_apply<3, 2, dev::FORM_ELAS, false, double>(p, 3, x, y, s);
    }
    return;
  }
  fail(DB2_ERR_UNSUPPORTED, "matrix-free action not provided for this form/element");
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
  const bool fp32 = precision == DB2_FP32_CONTRACT;
  if (precision != DB2_FP64 && !fp32) fail(DB2_ERR_ARGUMENT, "unknown precision %d", precision);
  dev::AsmParams p = make_params(P);
  p.kscale = a.f.coeff == DB2_COEFF_P1_SCALED ? a.f.constant[0] : 1.0;
  p.kappa = a.w;
  // L = kappa * f * v * dx contributes when its coefficient is P1_SCALED
  // (the kappa-weighted load); any other load does not depend on kappa.
  const bool loadk = gb && L.f.kind == DB2_FORM_LOAD && L.f.coeff == DB2_COEFF_P1_SCALED;
  if (loadk) {
    if (!L.w) fail(DB2_ERR_ARGUMENT, "kappa-weighted load needs its P1 field f");
    p.f = L.w;
    p.fc[0] = 1.0;
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
