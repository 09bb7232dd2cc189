// assemble.cuh -- device code of the row-gather assembly engine.
//
// Execution model (the B200 replacement of Assembler::assemble_cells,
// dolfin/fem/Assembler.cpp:148-193, with EigenMatrix::add,
// dolfin/la/EigenMatrix.cpp:156-166):
//
//   * one CTA per tile = a contiguous range of node rows of one test
//     component; the tile's CSR value segment is contiguous in HBM and is
//     accumulated in shared memory, then written once, coalesced;
//   * one thread per (node row, trial component block); it walks the cells
//     incident to its node in ascending cell order -- the order in which
//     DOLFIN's cell loop adds their contributions -- recomputes the affine
//     geometry in FP64, evaluates the node's element-matrix row as reference
//     tensor x geometry tensor, and adds it into its own row segment at the
//     precomputed column slots.  Rows never share slots, so the scatter is
//     deterministic without atomics.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "generated/element_rows.h"
#include "internal.h"

namespace db2 {
namespace dev {

enum { FORM_DIFF = 0, FORM_ELAS = 1 };
enum { LOAD_NONE = 0, LOAD_CONST = 1, LOAD_P1 = 2 };
constexpr int kMaxTileThreads = 256;

template <int D, int P>
struct El {
  static constexpr int NV = D + 1;
  static constexpr int NE = D == 3 ? 6 : 3;
  static constexpr int K = P == 1 ? NV : NV + NE;
  static constexpr int KP = (K + 3) / 4 * 4;
};

// ---- canonical relabelling ----------------------------------------------
// Packed permutation (2 bits per new vertex) that makes local node li
// canonical: vertex li first, or the endpoints of edge li first; the rest in
// ascending order.  Same rule as db2::canonical_perm on the host.
__host__ __device__ constexpr int edge_end(int D, int e, int s) {
  // TetrahedronCell.cpp:119-124 / TriangleCell.cpp:106-108 local edges
  if (D == 3) {
    switch (e) {
      case 0: return s ? 3 : 2;
      case 1: return s ? 3 : 1;
      case 2: return s ? 2 : 1;
      case 3: return s ? 3 : 0;
      case 4: return s ? 2 : 0;
      default: return s ? 1 : 0;
    }
  }
  switch (e) {
    case 0: return s ? 2 : 1;
    case 1: return s ? 2 : 0;
    default: return s ? 1 : 0;
  }
}
__host__ __device__ constexpr uint32_t perm_code(int D, int li) {
  int first0 = li, first1 = -1;
  if (li > D) {
    first0 = edge_end(D, li - D - 1, 0);
    first1 = edge_end(D, li - D - 1, 1);
  }
  int perm[4] = {0, 0, 0, 0};
  int n = 0;
  perm[n++] = first0;
  if (first1 >= 0) perm[n++] = first1;
  for (int a = 0; a <= D; ++a)
    if (a != first0 && a != first1) perm[n++] = a;
  uint32_t code = 0;
  for (int a = 0; a <= D; ++a) code |= uint32_t(perm[a]) << (2 * a);
  return code;
}
__host__ __device__ constexpr uint64_t perm_pack(int D, int lo) {
  uint64_t r = 0;
  const int K = D == 3 ? 10 : 6;
  for (int i = 0; i < 8; ++i)
    if (lo + i < K) r |= uint64_t(perm_code(D, lo + i)) << (8 * i);
  return r;
}
template <int D>
__device__ __forceinline__ uint32_t perm_of(int li) {
  constexpr uint64_t lo = perm_pack(D, 0), hi = perm_pack(D, 8);
  const uint64_t w = li < 8 ? (lo >> (8 * li)) : (hi >> (8 * (li - 8)));
  return uint32_t(w) & 0xffu;
}
template <typename T>
__device__ __forceinline__ T sel4(const T (&v)[4], uint32_t idx) {
  return idx == 0 ? v[0] : idx == 1 ? v[1] : idx == 2 ? v[2] : v[3];
}
template <typename T>
__device__ __forceinline__ T sel3(const T (&v)[3], uint32_t idx) {
  return idx == 0 ? v[0] : idx == 1 ? v[1] : v[2];
}

// ---- geometry (FP64) ------------------------------------------------------
// Barycentric gradients g[a] = grad(lambda_a) and |T| of the affine simplex
// with (relabelled) vertices x[0..D]: rows of J^-1 for a >= 1, g[0] = -sum.
template <int D>
struct Geometry {
  double g[D + 1][D];
  double vol;
};

__device__ __forceinline__ void geometry(const double (&x)[4][3], Geometry<3>& G) {
  double c[3][3];
  for (int m = 0; m < 3; ++m)
    for (int r = 0; r < 3; ++r) c[m][r] = x[m + 1][r] - x[0][r];
  double n[3][3];  // n[m] = c[m+1] x c[m+2]
  for (int m = 0; m < 3; ++m) {
    const double* a = c[(m + 1) % 3];
    const double* b = c[(m + 2) % 3];
    n[m][0] = a[1] * b[2] - a[2] * b[1];
    n[m][1] = a[2] * b[0] - a[0] * b[2];
    n[m][2] = a[0] * b[1] - a[1] * b[0];
  }
  const double det = c[0][0] * n[0][0] + c[0][1] * n[0][1] + c[0][2] * n[0][2];
  const double inv = __drcp_rn(det);
  for (int r = 0; r < 3; ++r) {
    G.g[1][r] = n[0][r] * inv;
    G.g[2][r] = n[1][r] * inv;
    G.g[3][r] = n[2][r] * inv;
    G.g[0][r] = -(G.g[1][r] + G.g[2][r] + G.g[3][r]);
  }
  G.vol = fabs(det) * (1.0 / 6.0);
}

__device__ __forceinline__ void geometry(const double (&x)[3][2], Geometry<2>& G) {
  const double c1x = x[1][0] - x[0][0], c1y = x[1][1] - x[0][1];
  const double c2x = x[2][0] - x[0][0], c2y = x[2][1] - x[0][1];
  const double det = c1x * c2y - c1y * c2x;
  const double inv = __drcp_rn(det);
  G.g[1][0] = c2y * inv;
  G.g[1][1] = -c2x * inv;
  G.g[2][0] = -c1y * inv;
  G.g[2][1] = c1x * inv;
  G.g[0][0] = -(G.g[1][0] + G.g[2][0]);
  G.g[0][1] = -(G.g[1][1] + G.g[2][1]);
  G.vol = fabs(det) * 0.5;
}

template <int D>
__device__ __forceinline__ double gdot(const Geometry<D>& G, int a, int b) {
  double s = G.g[a][0] * G.g[b][0];
  for (int r = 1; r < D; ++r) s = fma(G.g[a][r], G.g[b][r], s);
  return s;
}

// ---- generated reference-tensor rows ---------------------------------------
template <int D, int P, typename CT>
struct Rows;
#define DB2_ROWS(D_, P_, NAME, K_)                                                          \
  template <typename CT>                                                                   \
  struct Rows<D_, P_, CT> {                                                                \
    __device__ static void v_k1(const CT (&W)[1][D_ + 1], CT (&o)[K_]) {                    \
      gen::grad_grad_##NAME##_v_k1<CT>(W, o);                                               \
    }                                                                                      \
    __device__ static void v_kp1(const CT (&W)[1][D_ + 1], const CT (&k)[D_ + 1],           \
                                 CT (&o)[K_]) {                                            \
      gen::grad_grad_##NAME##_v_kp1<CT>(W, k, o);                                           \
    }                                                                                      \
    __device__ static double v_f1() { return gen::load_##NAME##_v_f1<double>(); }           \
    __device__ static double v_fp1(const double (&f)[D_ + 1]) {                             \
      return gen::load_##NAME##_v_fp1<double>(f);                                           \
    }                                                                                      \
    __device__ static void v_kfp1(const CT (&f)[D_ + 1], CT (&o)[D_ + 1]) {                 \
      gen::load_##NAME##_v_kfp1<CT>(f, o);                                                  \
    }
#define DB2_ROWS_EDGE(D_, NAME, K_)                                                         \
  __device__ static void e_k1(const CT (&W)[2][D_ + 1], CT (&o)[K_]) {                      \
    gen::grad_grad_##NAME##_e_k1<CT>(W, o);                                                 \
  }                                                                                        \
  __device__ static void e_kp1(const CT (&W)[2][D_ + 1], const CT (&k)[D_ + 1], CT (&o)[K_]) { \
    gen::grad_grad_##NAME##_e_kp1<CT>(W, k, o);                                             \
  }                                                                                        \
  __device__ static double e_f1() { return gen::load_##NAME##_e_f1<double>(); }             \
  __device__ static double e_fp1(const double (&f)[D_ + 1]) {                               \
    return gen::load_##NAME##_e_fp1<double>(f);                                             \
  }                                                                                        \
  __device__ static void e_kfp1(const CT (&f)[D_ + 1], CT (&o)[D_ + 1]) {                   \
    gen::load_##NAME##_e_kfp1<CT>(f, o);                                                    \
  }
DB2_ROWS(3, 1, p1tet, 4)
};
DB2_ROWS(3, 2, p2tet, 10)
DB2_ROWS_EDGE(3, p2tet, 10)
};
DB2_ROWS(2, 1, p1tri, 3)
};
DB2_ROWS(2, 2, p2tri, 6)
DB2_ROWS_EDGE(2, p2tri, 6)
};
#undef DB2_ROWS
#undef DB2_ROWS_EDGE

// ---- kernel parameters ------------------------------------------------------
struct AsmParams {
  const Tile* tiles;
  const int32_t* node_rowptr;
  const uint32_t* inc_ptr;
  const uint32_t* inc;
  const uint8_t* pos;
  const uint32_t* cells;
  const double* x;          // padded coordinates
  const uint32_t* cell_nodes;
  const uint32_t* cell_inc; // incidence index of (cell, local node)
  const double* kappa;      // P1 field (matrix form) or null
  double kscale;
  const double* f;          // P1 field (load form) or null
  double fc[3];
  double mu, lmbda;
  double* vals;
  double* b;
  int64_t nnz_node;
  int64_t nnodes;
  int add_values;
  const uint8_t* bc_flags;  // dof-level Dirichlet flags or null
  const double* bc_vals;
};

// Loads the relabelled vertices of cell `cell` for local node li.
template <int D>
__device__ __forceinline__ void load_cell(const AsmParams& p, uint32_t cell, int li,
                                          uint32_t (&pv)[D + 1], uint32_t& code) {
  code = perm_of<D>(li);
  if constexpr (D == 3) {
    const uint4 v4 = __ldg(reinterpret_cast<const uint4*>(p.cells) + cell);
    const uint32_t v[4] = {v4.x, v4.y, v4.z, v4.w};
    for (int a = 0; a < 4; ++a) pv[a] = sel4(v, (code >> (2 * a)) & 3u);
  } else {
    const uint32_t* c = p.cells + 3 * size_t(cell);
    const uint32_t v[3] = {__ldg(c), __ldg(c + 1), __ldg(c + 2)};
    for (int a = 0; a < 3; ++a) pv[a] = sel3(v, (code >> (2 * a)) & 3u);
  }
}

template <int D>
__device__ __forceinline__ void load_coords(const AsmParams& p, const uint32_t (&pv)[D + 1],
                                            double (&x)[D + 1][D]) {
  if constexpr (D == 3) {
    const double2* X = reinterpret_cast<const double2*>(p.x);
    for (int a = 0; a < 4; ++a) {
      const double2 xy = __ldg(X + 2 * size_t(pv[a]));
      const double2 zw = __ldg(X + 2 * size_t(pv[a]) + 1);
      x[a][0] = xy.x;
      x[a][1] = xy.y;
      x[a][2] = zw.x;
    }
  } else {
    const double2* X = reinterpret_cast<const double2*>(p.x);
    for (int a = 0; a < 3; ++a) {
      const double2 xy = __ldg(X + pv[a]);
      x[a][0] = xy.x;
      x[a][1] = xy.y;
    }
  }
}

// Element-matrix row of the canonical node (vertex 0 or edge (0,1)) for the
// trial component block e (test component c) into out[K] (contraction type CT).
template <int D, int P, int FORM, bool KP1, typename CT>
__device__ __forceinline__ void element_row(const AsmParams& p, const Geometry<D>& G,
                                            bool vertex, int c, int e,
                                            const double (&kap)[D + 1],
                                            CT (&out)[El<D, P>::K]) {
  using R = Rows<D, P, CT>;
  constexpr int NB = D + 1;
  CT kc[NB];
  if constexpr (KP1)
    for (int a = 0; a < NB; ++a) kc[a] = CT(kap[a]);
  auto wval = [&](int a, int b) -> double {
    if constexpr (FORM == FORM_DIFF) {
      return G.vol * gdot<D>(G, a, b) * p.kscale;
    } else {
      double gac = G.g[a][0], gae = G.g[a][0], gbc = G.g[b][0], gbe = G.g[b][0];
      for (int r = 1; r < D; ++r) {
        if (c == r) { gac = G.g[a][r]; gbc = G.g[b][r]; }
        if (e == r) { gae = G.g[a][r]; gbe = G.g[b][r]; }
      }
      double w = p.lmbda * gac * gbe + p.mu * gae * gbc;
      if (c == e) w = fma(p.mu, gdot<D>(G, a, b), w);
      return G.vol * w;
    }
  };
  if (P == 1 || vertex) {
    CT W[1][NB];
    for (int b = 0; b < NB; ++b) W[0][b] = CT(wval(0, b));
    if constexpr (KP1) R::v_kp1(W, kc, out);
    else R::v_k1(W, out);
  } else {
    if constexpr (P == 2) {
      CT W[2][NB];
      for (int a = 0; a < 2; ++a)
        for (int b = 0; b < NB; ++b) W[a][b] = CT(wval(a, b));
      if constexpr (KP1) R::e_kp1(W, kc, out);
      else R::e_k1(W, out);
    }
  }
}

template <int D, int P, int LOADM>
__device__ __forceinline__ double load_row(const AsmParams& p, const Geometry<D>& G, bool vertex,
                                           int c, const double (&fv)[D + 1]) {
  using R = Rows<D, P, double>;
  if constexpr (LOADM == LOAD_CONST) {
    double r;
    if constexpr (P == 2) r = vertex ? R::v_f1() : R::e_f1();
    else r = R::v_f1();
    return G.vol * r * p.fc[c];
  } else if constexpr (LOADM == LOAD_P1) {
    double r;
    if constexpr (P == 2) r = vertex ? R::v_fp1(fv) : R::e_fp1(fv);
    else r = R::v_fp1(fv);
    return G.vol * r * p.fc[0];
  } else {
    return 0.0;
  }
}

// One tile: rows [t.n0, t.n1) of test component t.comp.  `acc` holds the
// tile's CSR value segment.  Works for any blockDim >= units of the tile.
template <int D, int P, int FORM, bool KP1, int LOADM, typename CT>
__device__ __forceinline__ void tile_body(const AsmParams& p, const Tile t, double* acc) {
  using E = El<D, P>;
  constexpr int BS = FORM == FORM_ELAS ? D : 1;
  const int32_t r0 = __ldg(p.node_rowptr + t.n0), r1 = __ldg(p.node_rowptr + t.n1);
  const int seg = BS * (r1 - r0);
  for (int i = threadIdx.x; i < seg; i += blockDim.x) acc[i] = 0.0;
  __syncthreads();
  const int units = (t.n1 - t.n0) * BS;
  for (int u = threadIdx.x; u < units; u += blockDim.x) {
    const int node = t.n0 + u / BS;
    const int e = u % BS;
    const int32_t ra = __ldg(p.node_rowptr + node);
    const int32_t L = __ldg(p.node_rowptr + node + 1) - ra;
    double* my = acc + BS * (ra - r0) + e * L;
    const uint32_t i0 = __ldg(p.inc_ptr + node), i1 = __ldg(p.inc_ptr + node + 1);
    double bsum = 0.0;
    for (uint32_t ii = i0; ii < i1; ++ii) {
      const uint32_t word = __ldg(p.inc + ii);
      const uint32_t cell = word & 0x0fffffffu;
      const int li = int(word >> 28);
      const bool vertex = li <= D;
      uint32_t pv[D + 1], code;
      load_cell<D>(p, cell, li, pv, code);
      double x[D + 1][D];
      load_coords<D>(p, pv, x);
      double kap[D + 1];
      if constexpr (KP1)
        for (int a = 0; a <= D; ++a) kap[a] = __ldg(p.kappa + pv[a]);
      Geometry<D> G;
      geometry(x, G);
      CT out[E::K];
      element_row<D, P, FORM, KP1, CT>(p, G, vertex, t.comp, e, kap, out);
      const uint32_t* pw = reinterpret_cast<const uint32_t*>(p.pos + size_t(ii) * E::KP);
      uint32_t w[E::KP / 4];
      for (int q = 0; q < E::KP / 4; ++q) w[q] = __ldg(pw + q);
#pragma unroll
      for (int j = 0; j < E::K; ++j) {
        const uint32_t slot = (w[j >> 2] >> (8 * (j & 3))) & 0xffu;
        my[slot] += double(out[j]);
      }
      if constexpr (LOADM != LOAD_NONE) {
        if (e == 0) {
          double fv[D + 1];
          if constexpr (LOADM == LOAD_P1)
            for (int a = 0; a <= D; ++a) fv[a] = __ldg(p.f + pv[a]);
          bsum += load_row<D, P, LOADM>(p, G, vertex, t.comp, fv);
        }
      }
    }
    if constexpr (LOADM != LOAD_NONE) {
      if (e == 0) {
        double* bp = p.b + int64_t(t.comp) * p.nnodes + node;
        *bp = p.add_values ? *bp + bsum : bsum;
      }
    }
  }
  __syncthreads();
  double* dst = p.vals + int64_t(t.comp) * BS * p.nnz_node + int64_t(BS) * r0;
  if (p.add_values) {
    for (int i = threadIdx.x; i < seg; i += blockDim.x) dst[i] += acc[i];
  } else {
    for (int i = threadIdx.x; i < seg; i += blockDim.x) dst[i] = acc[i];
  }
  __syncthreads();
}

template <int D, int P, int FORM, bool KP1, int LOADM, typename CT>
__global__ void __launch_bounds__(kMaxTileThreads) k_assemble(const AsmParams p) {
  extern __shared__ double acc[];
  tile_body<D, P, FORM, KP1, LOADM, CT>(p, p.tiles[blockIdx.x], acc);
}

}  // namespace dev
}  // namespace db2
