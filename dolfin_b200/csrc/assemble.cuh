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
//   * an incidence record carries the relabelled cell's other vertices (as
//     offsets from the row's fixed vertex) and its column slots, so one
//     record load and two or three vertex-record loads feed an incidence;
//     records of 32 consecutive nodes are interleaved so that a warp's record
//     loads are contiguous.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <type_traits>

#include "generated/element_rows.h"
#include "internal.h"

namespace db2 {
namespace dev {

enum { FORM_DIFF = 0, FORM_ELAS = 1 };
// loads: none, constant f, P1 f, and kappa*f with the bilinear form's P1
// kappa (the kappa-weighted load whose derivative the adjoint also takes)
enum { LOAD_NONE = 0, LOAD_CONST = 1, LOAD_P1 = 2, LOAD_KP1 = 3 };
#ifndef DB2_TILE_MAX_THREADS
#define DB2_TILE_MAX_THREADS 256
#endif
constexpr int kMaxTileThreads = DB2_TILE_MAX_THREADS;

template <int D, int P>
struct El {
  static constexpr int NV = D + 1;
  static constexpr int NE = D == 3 ? 6 : 3;
  static constexpr int K = P == 1 ? NV : NV + NE;
  // incidence record: D int16 vertex offsets, then K slot bytes
  static constexpr int RS = 2 * D + K <= 8 ? 8 : 16;
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
// Relabelled local node j -> original local node for canonical node li,
// packed 4 bits per node (the device form of db2::canonical_node_map).
__host__ __device__ constexpr int cell_edge_of(int D, int a, int b) {
  for (int e = 0; e < (D == 3 ? 6 : 3); ++e) {
    const int p = edge_end(D, e, 0), q = edge_end(D, e, 1);
    if ((p == a && q == b) || (p == b && q == a)) return e;
  }
  return -1;
}
__host__ __device__ constexpr uint64_t node_map_code(int D, int P, int li) {
  const uint32_t pc = perm_code(D, li);
  int perm[4] = {0, 0, 0, 0};
  for (int a = 0; a <= D; ++a) perm[a] = int((pc >> (2 * a)) & 3u);
  const int nb = D + 1, ne = P == 2 ? (D == 3 ? 6 : 3) : 0;
  uint64_t code = 0;
  for (int j = 0; j < nb + ne; ++j) {
    const int o = j < nb ? perm[j]
                         : nb + cell_edge_of(D, perm[edge_end(D, j - nb, 0)], perm[edge_end(D, j - nb, 1)]);
    code |= uint64_t(o) << (4 * j);
  }
  return code;
}
// the code of a runtime li, by selection (no table in memory)
template <int D, int P>
__device__ __forceinline__ uint64_t node_map_of(int li) {
  constexpr int K = P == 1 ? D + 1 : (D == 3 ? 10 : 6);
  uint64_t m = node_map_code(D, P, 0);
#pragma unroll
  for (int q = 1; q < K; ++q)
    if (li == q) m = node_map_code(D, P, q);
  return m;
}

template <typename T>
__device__ __forceinline__ T sel4(const T (&v)[4], uint32_t idx) {
  return idx == 0 ? v[0] : idx == 1 ? v[1] : idx == 2 ? v[2] : v[3];
}
template <typename T>
__device__ __forceinline__ T sel3(const T (&v)[3], uint32_t idx) {
  return idx == 0 ? v[0] : idx == 1 ? v[1] : v[2];
}

// 1/x for x > 0: the hardware approximation refined by two Newton-Raphson
// steps y <- y + y (1 - x y) (each roughly doubles the correct bits), about
// 1 ulp; cheaper than the correctly rounded reciprocal.
__device__ __forceinline__ double rcp_nr(double x) {
  double y;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
  double e = fma(-x, y, 1.0);
  y = fma(y, e, y);
  e = fma(-x, y, 1.0);
  return fma(y, e, y);
}

// ---- geometry (FP64) ------------------------------------------------------
// For the affine simplex with (relabelled) vertices x[0..D]: the unnormalised
// barycentric gradients n[a] = det(J) * grad(lambda_a) (cofactor vectors of
// J = [x1-x0, x2-x0, ...], n[0] = -sum), s = 1 / (D! |det J|) and |T|.
// Then |T| grad(l_a).grad(l_b) = s * n[a].n[b]: the geometry tensor needs one
// reciprocal and no division of the gradients.
template <int D>
struct Geometry {
  double n[D + 1][D];
  double s;
  double vol;
};

__device__ __forceinline__ void geometry(const double (&x)[4][3], Geometry<3>& G) {
  double c[3][3];
#pragma unroll
  for (int m = 0; m < 3; ++m)
#pragma unroll
    for (int r = 0; r < 3; ++r) c[m][r] = x[m + 1][r] - x[0][r];
#pragma unroll
  for (int m = 0; m < 3; ++m) {  // n[m+1] = c[m+1] x c[m+2]
    const double* a = c[(m + 1) % 3];
    const double* b = c[(m + 2) % 3];
    G.n[m + 1][0] = a[1] * b[2] - a[2] * b[1];
    G.n[m + 1][1] = a[2] * b[0] - a[0] * b[2];
    G.n[m + 1][2] = a[0] * b[1] - a[1] * b[0];
  }
#pragma unroll
  for (int r = 0; r < 3; ++r) G.n[0][r] = -(G.n[1][r] + G.n[2][r] + G.n[3][r]);
  const double det = c[0][0] * G.n[1][0] + c[0][1] * G.n[1][1] + c[0][2] * G.n[1][2];
  const double ad = fabs(det);
  G.vol = ad * (1.0 / 6.0);
  G.s = rcp_nr(6.0 * ad);
}

__device__ __forceinline__ void geometry(const double (&x)[3][2], Geometry<2>& G) {
  const double c1x = x[1][0] - x[0][0], c1y = x[1][1] - x[0][1];
  const double c2x = x[2][0] - x[0][0], c2y = x[2][1] - x[0][1];
  const double det = c1x * c2y - c1y * c2x;
  G.n[1][0] = c2y;
  G.n[1][1] = -c2x;
  G.n[2][0] = -c1y;
  G.n[2][1] = c1x;
  G.n[0][0] = -(c2y - c1y);
  G.n[0][1] = -(c1x - c2x);
  const double ad = fabs(det);
  G.vol = ad * 0.5;
  G.s = rcp_nr(2.0 * ad);
}

template <int D>
__device__ __forceinline__ double ndot(const Geometry<D>& G, int a, int b) {
  double s = G.n[a][0] * G.n[b][0];
#pragma unroll
  for (int r = 1; r < D; ++r) s = fma(G.n[a][r], G.n[b][r], s);
  return s;
}

// ---- generated reference-tensor rows ---------------------------------------
template <int D, int P, typename CT>
struct Rows;
#define DB2_ROWS(D_, P_, NAME, K_)                                                          \
  template <typename CT>                                                                   \
  struct Rows<D_, P_, CT> {                                                                \
    static constexpr double sv_k1 = gen::grad_grad_##NAME##_v_k1_scale;                    \
    static constexpr double sv_kp1 = gen::grad_grad_##NAME##_v_kp1_scale;                  \
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
  static constexpr double se_k1 = gen::grad_grad_##NAME##_e_k1_scale;                      \
  static constexpr double se_kp1 = gen::grad_grad_##NAME##_e_kp1_scale;                    \
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

// The device node maps (node_map_code) agree with the host's canonical
// relabelling (db2::canonical_node_map, which the assembly plan's slots
// follow); checked on the host before a cell-wise launch.
inline void check_node_maps(int D, int deg) {
  const int K = deg == 1 ? D + 1 : (D == 3 ? 10 : 6);
  int map[10];
  for (int li = 0; li < K; ++li) {
    canonical_node_map(D, deg, li, map);
    for (int j = 0; j < K; ++j)
      if (int((node_map_code(D, deg, li) >> (4 * j)) & 15u) != map[j])
        fail(DB2_ERR_UNSUPPORTED, "device node map disagrees with the host's (li %d, j %d)", li, j);
  }
}

// ---- kernel parameters ------------------------------------------------------
struct AsmParams {
  const Tile* tiles;
  const int32_t* node_rowptr;
  const int32_t* cols;       // dof-level CSR column indices
  const uint32_t* inc_ptr;   // node -> incidence range (node-contiguous numbering)
  const uint32_t* inc;       // node-contiguous incidence words (cell | local node << 28)
  const unsigned char* rec;  // interleaved incidence records (El::RS bytes each)
  const uint32_t* rec_goff;  // first record of each block of 32 nodes
  const unsigned char* rec_first;  // record of each node's first incidence, by node
  const uint32_t* cells;
  const uint32_t* edge_v;    // P2: sorted endpoints of each edge node
  const double* xw;          // vertex records: 3D (x,y,z,kappa), 2D (x,y,kappa,f)
  const uint32_t* cell_nodes;
  const uint32_t* cell_inc;  // node-contiguous incidence index of (cell, local node)
  const double* kappa;       // P1 field (matrix form) or null
  double kscale;
  const double* f;           // P1 field (load form) or null
  double fc[3];
  double mu, lmbda;
  double* vals;
  double* b;
  int64_t nnz_node;
  int64_t nnodes;
  // output layout: value (c, k) of the CSR at vals[c * vstride + k - vbase],
  // b entry (c, node) at b[c * bstride + node - bbase] -- the full arrays
  // (vstride = bs nnz_node, bstride = nnodes, bases 0), or a rank's row
  // block of nodes [n0, n1) held alone (vstride = bs (rowptr[n1] -
  // rowptr[n0]), vbase = bs rowptr[n0], bstride = n1 - n0, bbase = n0)
  int64_t vstride, vbase, bstride, bbase;
  int64_t nverts;
  int add_values;
  const uint8_t* bc_flags;   // dof-level Dirichlet flags or null
  const double* bc_vals;
};

// ---- incidence records -----------------------------------------------------
template <int D, int P>
struct Rec {
  uint32_t w[El<D, P>::RS / 4];
  // offset k of a non-fixed vertex of the relabelled cell (sign-extended int16)
  __device__ __forceinline__ int32_t delta(int k) const {
    return int32_t(int16_t(uint16_t((w[k >> 1] >> (16 * (k & 1))) & 0xffffu)));
  }
  // edge-node rows: bit j set if this incidence is the first (in incidence
  // order) to touch local node j's slot; stored in the unused last offset
  __device__ __forceinline__ uint32_t first_mask() const {
    return (w[(D - 1) >> 1] >> (16 * ((D - 1) & 1))) & 0xffffu;
  }
  // column slot (within the row) of relabelled local node j
  __device__ __forceinline__ uint32_t slot(int j) const {
    const int b = 2 * D + j;
    return (w[b >> 2] >> (8 * (b & 3))) & 0xffu;
  }
  // Offsets that do not fit 16 bits (vertex numbering spread further than
  // 32767 within a cell) are stored as -32768: the vertices of such a
  // record are then read through the incidence word and the cell instead.
  static constexpr int32_t kEscape = -32768;
  __device__ __forceinline__ bool escaped(int nused) const {
    bool e = false;
#pragma unroll
    for (int k = 0; k < D; ++k)
      if (k < nused) e = e || delta(k) == kEscape;
    return e;
  }
};

template <int D, int P>
__device__ __forceinline__ uint32_t rec_index(const AsmParams& p, uint32_t node, uint32_t m) {
  return __ldg(p.rec_goff + (node >> 5)) + (node & 31u) + 32u * m;
}

template <int D, int P>
__device__ __forceinline__ Rec<D, P> load_rec_from(const unsigned char* base, uint32_t idx) {
  Rec<D, P> r;
  if constexpr (El<D, P>::RS == 16) {
    const uint4 v = __ldg(reinterpret_cast<const uint4*>(base) + idx);
    r.w[0] = v.x; r.w[1] = v.y; r.w[2] = v.z; r.w[3] = v.w;
  } else {
    const uint2 v = __ldg(reinterpret_cast<const uint2*>(base) + idx);
    r.w[0] = v.x; r.w[1] = v.y;
  }
  return r;
}

template <int D, int P>
__device__ __forceinline__ Rec<D, P> load_rec(const AsmParams& p, uint32_t idx) {
  return load_rec_from<D, P>(p.rec, idx);
}

// Relabelled vertex ids of a cell for local node li (vertex ids v[] as stored).
template <int D>
__device__ __forceinline__ void relabel(const uint32_t (&v)[D + 1], uint32_t code,
                                        uint32_t (&pv)[D + 1]) {
#pragma unroll
  for (int a = 0; a <= D; ++a) {
    const uint32_t k = (code >> (2 * a)) & 3u;
    if constexpr (D == 3) pv[a] = sel4(v, k);
    else pv[a] = sel3(v, k);
  }
}

template <int D>
__device__ __forceinline__ void load_verts(const AsmParams& p, uint32_t cell, uint32_t (&v)[D + 1]);

// Relabelled vertex ids of incidence `inc_index` from its incidence word
// (cell | local node << 28) and the cell's vertex list: the path of records
// whose offsets did not fit 16 bits.
template <int D>
__device__ __noinline__ void incidence_vertices(const AsmParams& p, uint32_t inc_index,
                                                uint32_t (&pv)[D + 1]) {
  const uint32_t w = __ldg(p.inc + inc_index);
  uint32_t v[D + 1];
  load_verts<D>(p, w & 0x0fffffffu, v);
  relabel<D>(v, perm_of<D>(int(w >> 28)), pv);
}

template <int D>
__device__ __forceinline__ void load_verts(const AsmParams& p, uint32_t cell, uint32_t (&v)[D + 1]) {
  if constexpr (D == 3) {
    const uint4 v4 = __ldg(reinterpret_cast<const uint4*>(p.cells) + cell);
    v[0] = v4.x; v[1] = v4.y; v[2] = v4.z; v[3] = v4.w;
  } else {
    const uint32_t* c = p.cells + 3 * size_t(cell);
    v[0] = __ldg(c); v[1] = __ldg(c + 1); v[2] = __ldg(c + 2);
  }
}

// One 256-bit read-only load of a vertex record.
__device__ __forceinline__ void ld_rec4(const double* ptr, double& a, double& b, double& c, double& d) {
  asm volatile("ld.global.nc.v4.f64 {%0,%1,%2,%3}, [%4];"
               : "=d"(a), "=d"(b), "=d"(c), "=d"(d)
               : "l"(ptr));
}

// Coordinates, kappa and f of one vertex (f from the vertex record in 2D,
// from the P1 array in 3D).
template <int D, bool FP1>
__device__ __forceinline__ void load_vertex(const AsmParams& p, uint32_t v, double (&x)[D],
                                            double& kap, double& f) {
  double r0, r1, r2, r3;
  ld_rec4(p.xw + 4 * size_t(v), r0, r1, r2, r3);
  if constexpr (D == 3) {
    x[0] = r0; x[1] = r1; x[2] = r2;
    kap = r3;
    f = FP1 ? __ldg(p.f + v) : 0.0;
  } else {
    x[0] = r0; x[1] = r1;
    kap = r2;
    f = r3;
  }
}

template <int D, bool FP1>
__device__ __forceinline__ void load_vertex_data(const AsmParams& p, const uint32_t (&pv)[D + 1],
                                                 double (&x)[D + 1][D], double (&kap)[D + 1],
                                                 double (&fv)[D + 1]) {
#pragma unroll
  for (int a = 0; a <= D; ++a) load_vertex<D, FP1>(p, pv[a], x[a], kap[a], fv[a]);
}

// The fixed vertices of a row: the vertex itself (vertex node) or the two
// sorted endpoints (edge node) -- relabelled local vertices 0 (and 1) of
// every incident cell.
template <int D>
struct RowFix {
  int nfix;
  uint32_t base;
  double x[2][D];
  double kap[2];
  double f[2];
};

template <int D, int P, bool FP1>
__device__ __forceinline__ RowFix<D> load_row_fix(const AsmParams& p, uint32_t node) {
  RowFix<D> r;
  if (P == 1 || node < uint64_t(p.nverts)) {
    r.nfix = 1;
    r.base = node;
    load_vertex<D, FP1>(p, node, r.x[0], r.kap[0], r.f[0]);
    r.x[1][0] = 0.0;
  } else {
    r.nfix = 2;
    const uint2 e = __ldg(reinterpret_cast<const uint2*>(p.edge_v) + (node - p.nverts));
    r.base = e.x;
    load_vertex<D, FP1>(p, e.x, r.x[0], r.kap[0], r.f[0]);
    load_vertex<D, FP1>(p, e.y, r.x[1], r.kap[1], r.f[1]);
  }
  return r;
}

// Same with the kind of row known at compile time (NFIX fixed vertices).
template <int D, int P, bool FP1, int NFIX>
__device__ __forceinline__ RowFix<D> load_row_fix_n(const AsmParams& p, uint32_t node) {
  RowFix<D> r;
  r.nfix = NFIX;
  if constexpr (NFIX == 1) {
    r.base = node;
    load_vertex<D, FP1>(p, node, r.x[0], r.kap[0], r.f[0]);
  } else {
    const uint2 e = __ldg(reinterpret_cast<const uint2*>(p.edge_v) + (node - p.nverts));
    r.base = e.x;
    load_vertex<D, FP1>(p, e.x, r.x[0], r.kap[0], r.f[0]);
    load_vertex<D, FP1>(p, e.y, r.x[1], r.kap[1], r.f[1]);
  }
  return r;
}

template <int D, int P, bool FP1, int NFIX, bool ESC>
__device__ __forceinline__ void record_cell_n(const AsmParams& p, const RowFix<D>& F,
                                              const Rec<D, P>& r, uint32_t inc_index,
                                              double (&x)[D + 1][D],
                                              double (&kap)[D + 1], double (&fv)[D + 1]) {
  uint32_t pv[D + 1] = {};
  const bool esc = ESC && r.escaped(D + 1 - NFIX);
  if (esc) incidence_vertices<D>(p, inc_index, pv);
#pragma unroll
  for (int a = 0; a <= D; ++a) {
    if (a < NFIX) {
#pragma unroll
      for (int q = 0; q < D; ++q) x[a][q] = F.x[a][q];
      kap[a] = F.kap[a];
      fv[a] = F.f[a];
    } else {
      const uint32_t v = esc ? pv[a] : uint32_t(int32_t(F.base) + r.delta(a - NFIX));
      load_vertex<D, FP1>(p, v, x[a], kap[a], fv[a]);
    }
  }
}

// Fixed vertices by id only: their records are loaded again with each
// incidence (L1 hits), so no coordinates stay live across the row walk.
struct RowFixId {
  uint32_t v[2];
};
template <int D, int P, int NFIX>
__device__ __forceinline__ RowFixId load_row_fix_id(const AsmParams& p, uint32_t node) {
  RowFixId r;
  if constexpr (NFIX == 1) {
    r.v[0] = r.v[1] = node;
  } else {
    const uint2 e = __ldg(reinterpret_cast<const uint2*>(p.edge_v) + (node - p.nverts));
    r.v[0] = e.x;
    r.v[1] = e.y;
  }
  return r;
}
template <int D, int P, bool FP1, int NFIX, bool ESC>
__device__ __forceinline__ void record_cell_id(const AsmParams& p, const RowFixId& F,
                                               const Rec<D, P>& r, uint32_t inc_index,
                                               double (&x)[D + 1][D],
                                               double (&kap)[D + 1], double (&fv)[D + 1]) {
  uint32_t pv[D + 1] = {};
  const bool esc = ESC && r.escaped(D + 1 - NFIX);
  if (esc) incidence_vertices<D>(p, inc_index, pv);
#pragma unroll
  for (int a = 0; a <= D; ++a) {
    const uint32_t v = a < NFIX ? F.v[a]
                       : esc    ? pv[a]
                                : uint32_t(int32_t(F.v[0]) + r.delta(a - NFIX));
    load_vertex<D, FP1>(p, v, x[a], kap[a], fv[a]);
  }
}

// The relabelled cell of one record: fixed vertices first, then the others.
template <int D, int P, bool FP1>
__device__ __forceinline__ void record_cell(const AsmParams& p, const RowFix<D>& F,
                                            const Rec<D, P>& r, uint32_t inc_index,
                                            double (&x)[D + 1][D],
                                            double (&kap)[D + 1], double (&fv)[D + 1]) {
  uint32_t pv[D + 1] = {};
  const bool esc = r.escaped(D + 1 - F.nfix);
  if (esc) incidence_vertices<D>(p, inc_index, pv);
#pragma unroll
  for (int a = 0; a <= D; ++a) {
    if (a < F.nfix) {
#pragma unroll
      for (int q = 0; q < D; ++q) x[a][q] = F.x[a][q];
      kap[a] = F.kap[a];
      fv[a] = F.f[a];
    } else {
      const uint32_t v = esc ? pv[a] : uint32_t(int32_t(F.base) + r.delta(a - F.nfix));
      load_vertex<D, FP1>(p, v, x[a], kap[a], fv[a]);
    }
  }
}

// Element-matrix row of the canonical node (vertex 0 or edge (0,1)) for the
// trial component block e (test component c) into out[K] (contraction type CT):
// the FP64 geometry tensor W is formed, rounded to CT, and contracted with the
// generated reference tensor in CT.
template <int D, int P, int FORM, bool KP1, typename CT>
__device__ __forceinline__ void element_row(const AsmParams& p, const Geometry<D>& G,
                                            bool vertex, int c, int e,
                                            const double (&kap)[D + 1],
                                            CT (&out)[El<D, P>::K]) {
  using R = Rows<D, P, CT>;
  constexpr int NB = D + 1;
  CT kc[NB];
  if constexpr (KP1) {
#pragma unroll
    for (int a = 0; a < NB; ++a) kc[a] = CT(kap[a]);
  }
  // the generated rows take W times their scale (integer coefficients remain)
  double sig = KP1 ? R::sv_kp1 : R::sv_k1;
  if constexpr (P == 2) {
    if (!vertex) sig = KP1 ? R::se_kp1 : R::se_k1;
  }
  // elasticity: components c and e of every cofactor vector, selected once
  // per incidence rather than inside each entry of W^{ce}
  double nc[NB], ne[NB];
  if constexpr (FORM == FORM_ELAS) {
#pragma unroll
    for (int a = 0; a < NB; ++a) {
      nc[a] = G.n[a][0];
      ne[a] = G.n[a][0];
#pragma unroll
      for (int r = 1; r < D; ++r) {
        if (c == r) nc[a] = G.n[a][r];
        if (e == r) ne[a] = G.n[a][r];
      }
    }
  }
  auto wval = [&](int a, int b) -> double {
    if constexpr (FORM == FORM_DIFF) {
      return ndot<D>(G, a, b) * (G.s * (p.kscale * sig));
    } else {
      double w = p.lmbda * nc[a] * ne[b] + p.mu * ne[a] * nc[b];
      if (c == e) w = fma(p.mu, ndot<D>(G, a, b), w);
      return (G.s * sig) * w;
    }
  };
  if (P == 1 || vertex) {
    CT W[1][NB];
#pragma unroll
    for (int b = 0; b < NB; ++b) W[0][b] = CT(wval(0, b));
    if constexpr (KP1) R::v_kp1(W, kc, out);
    else R::v_k1(W, out);
  } else {
    if constexpr (P == 2) {
      CT W[2][NB];
#pragma unroll
      for (int a = 0; a < 2; ++a)
#pragma unroll
        for (int b = 0; b < NB; ++b) W[a][b] = CT(wval(a, b));
      if constexpr (KP1) R::e_kp1(W, kc, out);
      else R::e_k1(W, out);
    }
  }
}

template <int D, int P, int LOADM>
__device__ __forceinline__ double load_row(const AsmParams& p, const Geometry<D>& G, bool vertex,
                                           int c, const double (&fv)[D + 1],
                                           const double (&kap)[D + 1]) {
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
  } else if constexpr (LOADM == LOAD_KP1) {
    // int kappa f phi_i = sum_m kappa_m int lambda_m f phi_i (kappa P1)
    double o[D + 1];
    if constexpr (P == 2) {
      if (vertex) R::v_kfp1(fv, o);
      else R::e_kfp1(fv, o);
    } else {
      R::v_kfp1(fv, o);
    }
    double r = kap[0] * o[0];
#pragma unroll
    for (int m = 1; m <= D; ++m) r = fma(kap[m], o[m], r);
    return G.vol * r * p.fc[0];
  } else {
    return 0.0;
  }
}


// One row unit (node row, trial block e) of a tile whose rows are all vertex
// nodes (NFIX = 1 fixed vertex) or all edge nodes (NFIX = 2).
// Variant flags of the tile kernel (separate instantiations, so that the
// common case pays for neither): records with escaped vertex offsets, and
// Dirichlet data (without it the row walk carries no boundary-condition state).
enum { VAR_ESC = 1, VAR_BC = 2 };

template <int D, int P, int FORM, bool KP1, int LOADM, typename CT, int NFIX, int VAR>
__device__ __forceinline__ void row_unit(const AsmParams& p, const Tile& t, CT* acc,
                                         double* bpart, int32_t r0, int u) {
  using E = El<D, P>;
  constexpr int BS = FORM == FORM_ELAS ? D : 1;
  constexpr bool FP1 = LOADM == LOAD_P1 || LOADM == LOAD_KP1;
  constexpr bool vertex = NFIX == 1;
  constexpr bool ESC = (VAR & VAR_ESC) != 0;
  const bool bc = (VAR & VAR_BC) != 0 && p.bc_flags != nullptr;
  const uint32_t node = t.n0 + u / BS;
  const int e = u % BS;
  const int32_t ra = __ldg(p.node_rowptr + node);
  const int32_t L = __ldg(p.node_rowptr + node + 1) - ra;
  CT* my = acc + BS * (ra - r0) + e * L;
  const uint32_t i0 = __ldg(p.inc_ptr + node);
  const uint32_t cnt = __ldg(p.inc_ptr + node + 1) - i0;
  const uint32_t rbase = __ldg(p.rec_goff + (node >> 5)) + (node & 31u);
  double bsum = 0.0;
  const int64_t rowdof = int64_t(t.comp) * p.nnodes + node;
  bool row_bc = false;
  double row_g = 0.0;
  const int32_t* colrow = nullptr;
  if (bc) {
    row_bc = __ldg(p.bc_flags + rowdof) != 0;
    row_g = row_bc ? __ldg(p.bc_vals + rowdof) : 0.0;
    colrow = p.cols + int64_t(t.comp) * BS * p.nnz_node + int64_t(BS) * ra + e * L;
  }
  // Elasticity rows reload their fixed vertices with every incidence (L1
  // hits); the Poisson rows keep them in registers (measured on B200:
  // reloading costs 10 % on P2 Poisson; elasticity with first-touch stores at
  // 96 registers: 1.20 ms reloading against 1.32 keeping them).
  constexpr bool RELOAD = FORM == FORM_ELAS;
  using Fix = typename std::conditional<RELOAD, RowFixId, RowFix<D>>::type;
  Fix F;
  if constexpr (RELOAD) F = load_row_fix_id<D, P, NFIX>(p, node);
  else F = load_row_fix_n<D, P, FP1, NFIX>(p, node);
  // The unit owns acc[my, my + L) alone (the units' segments partition the
  // tile's), so it clears its own segment: no block barrier before the row
  // walk, whose first loads are already in flight.
  // Edge-node rows need no clearing: every slot of the row is written first
  // by a plain store, at the incidence the record marks as its first (fewer
  // shared-memory loads: P2 tets n=96 1.13 ms against 1.23, vector P2
  // elasticity n=48 1.20 against 1.28).
  constexpr bool FIRSTF = NFIX == 2;
  if (!FIRSTF || cnt == 0)
    for (int32_t k = 0; k < L; ++k) my[k] = CT(0);
  // The row node is relabelled local node 0 (vertex) or K-1 (edge (0,1)),
  // and an edge's end vertices are local nodes 0 and 1: these NREG columns
  // are the same for every incidence, so they are summed in registers (in
  // incidence order, as the segment would) and added once at the end.
  constexpr int NREG = vertex ? 1 : 3;
  constexpr int jstar = vertex ? 0 : E::K - 1;
  auto regcol = [](int i) { return i == 0 ? jstar : i - 1; };
  double rsum[NREG];
  uint32_t rslot[NREG];
#pragma unroll
  for (int i = 0; i < NREG; ++i) {
    rsum[i] = 0.0;
    rslot[i] = 0;
  }
  // the next record is fetched one incidence ahead: its load (the head of
  // the dependent chain record -> vertex records -> geometry) overlaps the
  // current incidence's arithmetic.  The first comes from the node-indexed
  // copy, so it is issued beside the row's other loads, not after rec_goff.
  Rec<D, P> rn{};
  if (cnt > 0) rn = load_rec_from<D, P>(p.rec_first, node);
  for (uint32_t m = 0; m < cnt; ++m) {
    const Rec<D, P> r = rn;
    if (m + 1 < cnt) rn = load_rec<D, P>(p, rbase + 32u * (m + 1));
    double x[D + 1][D], kap[D + 1], fv[D + 1];
    if constexpr (RELOAD) record_cell_id<D, P, FP1, NFIX, ESC>(p, F, r, i0 + m, x, kap, fv);
    else record_cell_n<D, P, FP1, NFIX, ESC>(p, F, r, i0 + m, x, kap, fv);
    Geometry<D> G;
    geometry(x, G);
    CT out[E::K];
    element_row<D, P, FORM, KP1, CT>(p, G, vertex, t.comp, e, kap, out);
    if constexpr (LOADM != LOAD_NONE) {
      if (e == 0) bsum += load_row<D, P, LOADM>(p, G, vertex, t.comp, fv, kap);
    }
    if (bc) {
      if (row_bc) {
#pragma unroll
        for (int j = 0; j < E::K; ++j) out[j] = CT((e == t.comp && j == jstar) ? 1 : 0);
        if constexpr (LOADM != LOAD_NONE) {
          if (e == 0) bsum = bsum - load_row<D, P, LOADM>(p, G, vertex, t.comp, fv, kap) + row_g;
        }
      } else {
#pragma unroll
        for (int j = 0; j < E::K; ++j) {
          const int32_t dof = __ldg(colrow + r.slot(j));
          if (__ldg(p.bc_flags + dof)) {
            bsum -= double(out[j]) * __ldg(p.bc_vals + dof);
            out[j] = CT(0);
          }
        }
      }
    }
#pragma unroll
    for (int i = 0; i < NREG; ++i) {
      rslot[i] = r.slot(regcol(i));
      rsum[i] += double(out[regcol(i)]);
    }
    // The slots of one incidence are distinct (the cell's nodes are distinct
    // columns of the row), so every segment load of the incidence is issued
    // before its first store: one shared-memory round trip per incidence
    // rather than one per column, which the compiler cannot arrange itself
    // (it cannot see that the addresses differ).
    const uint32_t fm = FIRSTF ? r.first_mask() : 0u;
    auto in_reg = [&](int j) {
      bool f = false;
#pragma unroll
      for (int i = 0; i < NREG; ++i) f = f || j == regcol(i);
      return f;
    };
    CT o[E::K];
#pragma unroll
    for (int j = 0; j < E::K; ++j) {
      o[j] = CT(0);
      if (!in_reg(j) && !(fm >> j & 1u)) o[j] = my[r.slot(j)];  // first touch: no load
    }
#pragma unroll
    for (int j = 0; j < E::K; ++j)
      if (!in_reg(j)) my[r.slot(j)] = o[j] + out[j];
  }
  if (cnt) {
#pragma unroll
    for (int i = 0; i < NREG; ++i) {
      if (FIRSTF) my[rslot[i]] = CT(0.0 + rsum[i]);  // no other write reaches these slots
      else my[rslot[i]] = CT(double(my[rslot[i]]) + rsum[i]);
    }
  }
  bpart[u] = bsum;
}

// Bulk copy shared -> global (cp.async.bulk, no tensor map): both addresses
// 16-byte aligned, bytes a multiple of 16.  Completion of the reads of the
// shared source is awaited by bulk_wait_read; the global writes are
// performed before the kernel completes.
__device__ __forceinline__ void bulk_fence() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void bulk_store(double* gdst, const double* ssrc, uint32_t bytes) {
  asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;\n\t"
               "cp.async.bulk.commit_group;"
               :
               : "l"(gdst), "r"(static_cast<uint32_t>(__cvta_generic_to_shared(ssrc))), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void bulk_wait_read() {
  asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
}

// One tile: rows [t.n0, t.n1) of test component t.comp.  `acc` holds the
// tile's CSR value segment (in the contraction type: the FP32-contraction
// path also accumulates in FP32 -- about 1e-7 of the row's largest entry,
// the columns kept in registers summed in FP64) followed by one double per
// row unit (load-vector partials).  blockDim must be at least the tile's unit
// count.
//
// With Dirichlet data (p.bc_flags) each element row is modified as
// SystemAssembler::apply_bc (dolfin/fem/SystemAssembler.cpp:1037-1070) does
// per cell: a Dirichlet row keeps only 1 on its diagonal and contributes g_i
// to b; other rows move their Dirichlet-column entries to b (b_i -= A_ij g_j)
// and zero them.
template <int D, int P, int FORM, bool KP1, int LOADM, typename CT, int VAR = VAR_BC>
__device__ __forceinline__ void tile_body(const AsmParams& p, const Tile t, double* acc) {
  constexpr int BS = FORM == FORM_ELAS ? D : 1;
  constexpr bool F64 = sizeof(CT) == 8;
  const int32_t r0 = __ldg(p.node_rowptr + t.n0), r1 = __ldg(p.node_rowptr + t.n1);
  const int seg = BS * (r1 - r0);
  double* dst = p.vals + int64_t(t.comp) * p.vstride + int64_t(BS) * r0 - p.vbase;
  // An FP64 segment is staged at the address parity (mod 16 bytes) of its
  // destination, so that its 16-byte-aligned middle leaves shared memory by
  // one bulk copy (the launch gives one double of slack for the shift).
  const int sh = F64 ? int((reinterpret_cast<uintptr_t>(dst) >> 3) & 1u) : 0;
  CT* segm = reinterpret_cast<CT*>(acc) + sh;
  double* bpart = acc + (sh + seg * int(sizeof(CT)) / 8 + 1);
  const int units = (t.n1 - t.n0) * BS;
  if (int(threadIdx.x) < units) {
    // tiles never mix vertex and edge nodes (the host cuts P2 tiles at the
    // first edge node), so the row kind is uniform over the block
    if (P == 1 || t.n0 < p.nverts)
      row_unit<D, P, FORM, KP1, LOADM, CT, 1, VAR>(p, t, segm, bpart, r0, int(threadIdx.x));
    else if constexpr (P == 2)
      row_unit<D, P, FORM, KP1, LOADM, CT, 2, VAR>(p, t, segm, bpart, r0, int(threadIdx.x));
  }
  // the segment's generic-proxy writes are made visible to the bulk copy
  // (async proxy) by this fence and the barrier
  if constexpr (F64) bulk_fence();
  __syncthreads();
  if constexpr (LOADM != LOAD_NONE) {
    // b of each row: its trial blocks' partials in block order
    for (int i = threadIdx.x; i < t.n1 - t.n0; i += blockDim.x) {
      double s = 0.0;
#pragma unroll
      for (int e = 0; e < BS; ++e) s += bpart[i * BS + e];
      double* bp = p.b + int64_t(t.comp) * p.bstride + (t.n0 - p.bbase) + i;
      *bp = p.add_values ? *bp + s : s;
    }
  }
  if (p.add_values) {
    for (int i = threadIdx.x; i < seg; i += blockDim.x) dst[i] += double(segm[i]);
  } else if constexpr (!F64) {
    for (int i = threadIdx.x; i < seg; i += blockDim.x) dst[i] = double(segm[i]);
  } else {
    // an unaligned first and last double by plain stores, the rest (16-byte
    // aligned at both ends, a multiple of 16 bytes) by one bulk copy that
    // thread 0 issues and waits to have read before the segment is reused
    const int nb = seg > sh ? (seg - sh) & ~1 : 0;
    if (threadIdx.x == 0 && nb > 0) bulk_store(dst + sh, segm + sh, uint32_t(nb) * 8u);
    if (threadIdx.x == blockDim.x - 1) {
      if (sh && seg > 0) dst[0] = segm[0];
      if (seg > sh + nb) dst[seg - 1] = segm[seg - 1];
    }
    if (threadIdx.x == 0 && nb > 0) bulk_wait_read();
  }
  __syncthreads();
}

// Register cap of the tile kernel (threads per CTA are chosen per pattern,
// 32..256, so the cap is given directly rather than through launch bounds).
// The kernel is latency bound, so resident warps per SM matter: with 64-thread
// tiles, 96 registers give 10 CTAs per SM against 8 at the ~120 the P2 rows
// take uncapped.  Measured on B200 (ms per A+b step): vector P2 elasticity
// n=48 1.346 against 1.373 (uncapped within 128), P2 tets n=96 1.304 against
// 1.325, P1 tets n=96 0.237 against 0.265; 104 registers was slower on the P2
// rows, 88 no faster, 80 spills.  The elasticity rows (first-touch stores,
// fixed vertices reloaded) take 96 too: 1.20 ms against 1.35 at 88.  The
// FP32-contraction rows keep fewer
// values live and take 80 (12 CTAs): 1.03-1.05x their time at 96 on the
// elasticity and P1 workloads, no change on P2 n=96.  The instantiations
// without Dirichlet data fit lower caps without spills (P2 88, elasticity
// 80) but are no faster there: P2 n=96 1.042-1.050 ms at 88 and 96,
// elasticity n=48 1.041 at 80 against 1.006 at 96.
#ifndef DB2_TILE_MAXNREG_P1
#define DB2_TILE_MAXNREG_P1 96
#endif
#ifndef DB2_TILE_MAXNREG_P2
#define DB2_TILE_MAXNREG_P2 96
#endif
#ifndef DB2_TILE_MAXNREG_F32
#define DB2_TILE_MAXNREG_F32 80
#endif
#ifndef DB2_TILE_MAXNREG_ELAS
#define DB2_TILE_MAXNREG_ELAS 96
#endif
template <int P, int FORM, typename CT>
constexpr int tile_maxnreg() {
  return sizeof(CT) == 4       ? DB2_TILE_MAXNREG_F32
         : FORM == FORM_ELAS ? DB2_TILE_MAXNREG_ELAS
         : P == 1            ? DB2_TILE_MAXNREG_P1
                             : DB2_TILE_MAXNREG_P2;
}
// VAR: VAR_ESC when the pattern has records whose vertex offsets did not fit
// 16 bits, VAR_BC when the call has Dirichlet data.
template <int D, int P, int FORM, bool KP1, int LOADM, typename CT, int VAR>
__global__ void __maxnreg__((tile_maxnreg<P, FORM, CT>())) k_assemble(const AsmParams p) {
  extern __shared__ __align__(16) double acc[];
  tile_body<D, P, FORM, KP1, LOADM, CT, VAR>(p, p.tiles[blockIdx.x], acc);
}

}  // namespace dev
}  // namespace db2
