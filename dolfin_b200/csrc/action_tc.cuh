// action_tc.cuh -- the FP32-contraction matrix-free action of
// kappa*inner(grad(u), grad(v))*dx on P2 tetrahedra, with the reference
// tensor x geometry tensor contraction on the tensor cores (tcgen05).
//
// Per cell K (Kirby & Logg's factorisation, the tensor of
// codegen/gen_reference_tensor.py):
//
//     A_K = G_K R / 60,   G_K[(m, ab)] = kappa_m |K| g_a.g_b  (40 features),
//
// R the exact integer reference tensor (40 x 55 symmetric entries, |R| <=
// 48).  A tile of 128 cells is one tensor-core product [128 x 80] x [80 x 64]
// -> FP32 in tensor memory: the geometry operand is computed in FP64 per
// cell, scaled by a power of two and split into two half-precision limbs
// (G = h1 + h2 2^-11, 22 significant bits; the features themselves in FP32
// from the FP64 geometry), the second limb's rows of R
// scaled by 2^-11 (exact in half precision), so the products are exact and
// the only rounding is the FP32 accumulation (~3e-7 of max |A_K|).  Each
// thread then reads its cell's 55 entries from tensor memory, forms
// y_K = A_K x_K in FP32 and writes y_K (FP32) to the cell's incidence
// slots; the ordered per-row gather sums them in FP64.
//
// One CTA = one warpgroup = 128 threads = 128 tensor-memory lanes (thread t
// <-> cell t of the tile <-> lane t); persistent over tiles.
#pragma once

#include <cuda_fp16.h>

#include "generated/ref_tensor.h"
#include "umma.cuh"

namespace db2 {
namespace dev {

constexpr int kTcM = 128;            // cells per tile: TMEM lanes and threads
constexpr int kTcF = 40;             // features kappa_m W_ab
constexpr int kTcK = 2 * kTcF;       // two half-precision limbs each
constexpr int kTcN = 64;             // 55 symmetric entries of A_K, padded
constexpr int kTcChunks = kTcK / 8;  // 16-byte K chunks (8 halves)
constexpr int kTcEntries = 55;
constexpr uint32_t kTcWaitLimit = 1u << 24;

// Operands in the canonical K-major layout without swizzle (umma.cuh):
// element (row, k) at a[k / 8][row], half k % 8 of that 16-byte cell, so
// 8 consecutive rows form a core matrix (SBO = 128 B) and consecutive K
// chunks are LBO = rows * 16 B apart.
struct TcSmem {
  uint4 a[kTcChunks][kTcM];  // geometry operand, one row per cell (20 KB)
  uint4 b[kTcChunks][kTcN];  // reference tensor, one row per entry (10 KB)
  unsigned long long bar;    // mbarrier: tensor-core products done
  uint32_t tmem;             // tensor-memory base of the accumulators
};

// Set when a tensor-core wait ran out (the outputs of that launch are NaN).
__device__ int g_tc_status = 0;

template <bool KP1>
__global__ void __launch_bounds__(kTcM, 5) k_apply_tc_p2(const AsmParams p, int64_t ncells,
                                                       const double* __restrict__ xin,
                                                       float* __restrict__ ycell) {
  extern __shared__ __align__(128) unsigned char tc_smem_raw[];
  TcSmem& S = *reinterpret_cast<TcSmem*>(tc_smem_raw);
  const int t = threadIdx.x, warp = t >> 5;
  // B: the generated operand (entry n = (i <= j) row-major, limb-2 rows
  // scaled by 2^-11), copied to shared memory
  for (int idx = t; idx < kTcChunks * kTcN; idx += kTcM)
    (&S.b[0][0])[idx] = __ldg(&gen::kRefP2TetB[0][0] + idx);
  const uint32_t bar = umma::smem_u32(&S.bar);
  if (t == 0) umma::mbar_init(bar, 1);
  if (warp == 0) umma::tmem_alloc(umma::smem_u32(&S.tmem), kTcN);
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  const uint32_t tmem = S.tmem;
  constexpr uint32_t idesc = umma::idesc_f16_f32(kTcM, kTcN);
  const int64_t ntiles = (ncells + kTcM - 1) / kTcM;
  uint32_t phase = 0;
  // the cell data of a thread's next tile is loaded one tile ahead: vertex
  // ids and edge nodes do not depend on the arithmetic (the incidence slots
  // are loaded where they are used: 5 CTAs per SM need <= 102 registers)
  const int64_t stride = int64_t(gridDim.x) * kTcM;
  uint4 nv4 = make_uint4(0, 0, 0, 0);
  uint32_t nnode[6] = {0, 0, 0, 0, 0, 0};
  auto prefetch = [&](int64_t c) {
    if (c < ncells) {
      nv4 = __ldg(reinterpret_cast<const uint4*>(p.cells) + c);
#pragma unroll
      for (int j = 0; j < 6; ++j) nnode[j] = __ldg(p.cell_nodes + size_t(c) * 10 + 4 + j);
    }
  };
  prefetch(int64_t(blockIdx.x) * kTcM + t);
  for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int64_t cell = tile * kTcM + t;
    const bool live = cell < ncells;
    const uint4 v4 = nv4;
    uint32_t nodes[10];
    nodes[0] = v4.x;
    nodes[1] = v4.y;
    nodes[2] = v4.z;
    nodes[3] = v4.w;
#pragma unroll
    for (int j = 0; j < 6; ++j) nodes[4 + j] = nnode[j];
    prefetch(cell + stride);
    // ---- geometry operand: FP64 geometry, FP32 features, two half limbs ------
    uint32_t hp[kTcK / 2];  // packed half pairs, k = 2i, 2i + 1
    float xv[10];
    int e = 0;
    if (live) {
      double x[4][3], kap[4];
#pragma unroll
      for (int a = 0; a < 4; ++a) {
        double f;
        load_vertex<3, false>(p, nodes[a], x[a], kap[a], f);
      }
#pragma unroll
      for (int j = 0; j < 10; ++j) xv[j] = float(__ldg(xin + nodes[j]));
      Geometry<3> Gm;
      geometry(x, Gm);
      float W[10], km[4];
      float wmax = 0.f, kmax = 0.f;
      int q = 0;
#pragma unroll
      for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = a; b < 4; ++b, ++q) {
          W[q] = float(Gm.s * ndot<3>(Gm, a, b));  // |K| g_a.g_b
          wmax = fmaxf(wmax, fabsf(W[q]));
        }
#pragma unroll
      for (int m = 0; m < 4; ++m) {
        km[m] = float(KP1 ? p.kscale * kap[m] : p.kscale);
        kmax = fmaxf(kmax, fabsf(km[m]));
      }
      // |G| < 2^e; the operand is G 2^-e (a power of two: exact)
      frexpf(wmax * kmax, &e);
      e = max(-120, min(120, e));
      const float sc = __int_as_float((127 - e) << 23);
      float g[kTcF];
#pragma unroll
      for (int m = 0; m < 4; ++m)
#pragma unroll
        for (int r = 0; r < 10; ++r) g[m * 10 + r] = km[m] * W[r] * sc;
#pragma unroll
      for (int i = 0; i < kTcF / 2; ++i) {
        const __half2 h1 = __floats2half2_rn(g[2 * i], g[2 * i + 1]);
        const float2 back = __half22float2(h1);
        const __half2 h2 = __floats2half2_rn((g[2 * i] - back.x) * 2048.f, (g[2 * i + 1] - back.y) * 2048.f);
        hp[i] = *reinterpret_cast<const uint32_t*>(&h1);
        hp[kTcF / 2 + i] = *reinterpret_cast<const uint32_t*>(&h2);
      }
    } else {
#pragma unroll
      for (int i = 0; i < kTcK / 2; ++i) hp[i] = 0u;
    }
#pragma unroll
    for (int c = 0; c < kTcChunks; ++c) S.a[c][t] = make_uint4(hp[4 * c], hp[4 * c + 1], hp[4 * c + 2], hp[4 * c + 3]);
    // the tile's rows (generic proxy) -> the tensor core (async proxy); the
    // previous tile's tensor-memory reads are complete before the product
    umma::fence_async_smem();
    umma::fence_before_sync();
    __syncthreads();
    if (t == 0) {
      umma::fence_after_sync();
#pragma unroll
      for (int s = 0; s < kTcK / 16; ++s) {
        const uint64_t ad = umma::desc_kmajor(umma::smem_u32(&S.a[2 * s][0]), kTcM * 16, 128);
        const uint64_t bd = umma::desc_kmajor(umma::smem_u32(&S.b[2 * s][0]), kTcN * 16, 128);
        umma::mma_f16(tmem, ad, bd, idesc, s > 0 ? 1u : 0u);
      }
      umma::commit(bar);
    }
    const bool done = __syncthreads_and(umma::mbar_wait(bar, phase, kTcWaitLimit));
    phase ^= 1u;
    if (!done) {
      if (t == 0) atomicExch(&g_tc_status, 1);
      if (live)
        for (int j = 0; j < 10; ++j) ycell[__ldg(p.cell_inc + size_t(cell) * 10 + j)] = __int_as_float(-1);
      break;
    }
    umma::fence_after_sync();
    float acc[64];
    umma::tmem_ld64(tmem + (uint32_t(warp * 32) << 16), acc);
    if (live) {
      float y[10];
#pragma unroll
      for (int j = 0; j < 10; ++j) y[j] = 0.f;
      int n = 0;
#pragma unroll
      for (int i = 0; i < 10; ++i)
#pragma unroll
        for (int j = i; j < 10; ++j, ++n) {
          y[i] = fmaf(acc[n], xv[j], y[i]);
          if (j != i) y[j] = fmaf(acc[n], xv[i], y[j]);
        }
      const float sc = __int_as_float((127 + e) << 23) * (1.f / float(gen::kRefP2TetDen));
#pragma unroll
      for (int j = 0; j < 10; ++j) ycell[__ldg(p.cell_inc + size_t(cell) * 10 + j)] = y[j] * sc;
    }
  }
  umma::fence_before_sync();
  __syncthreads();
  if (warp == 0) {
    umma::fence_after_sync();
    umma::tmem_free(tmem, kTcN);
  }
}

}  // namespace dev
}  // namespace db2
