// launch.cuh -- shared launch helpers for the assembly kernel instantiations.
#pragma once

#include <vector>

#include "assemble.cuh"

namespace db2 {
namespace dev {

struct LaunchCfg {
  const std::vector<int32_t>* class_begin;  // tile ranges launched together
  const std::vector<int32_t>* class_smem;
  int threads;
  cudaStream_t stream;
  bool escapes = false;  // the pattern has records with escaped vertex offsets
};

// Let `kern` use all the dynamic shared memory the current device allows a
// block, less the kernel's own static shared memory (the opt-in limit covers
// both).  Done once per kernel and device; `done` is the caller's per-kernel
// record of the devices already configured.
template <typename Kernel>
void allow_dynamic_smem(Kernel kern, unsigned long long& done) {
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 64 && (done >> dev & 1ull)) return;
  int optin = 0;
  cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  cudaFuncAttributes fa{};
  cudaFuncGetAttributes(&fa, kern);
  cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       optin - int(fa.sharedSizeBytes));
  check_cuda("shared-memory allowance");
  if (dev < 64) done |= 1ull << dev;
}

#ifndef DB2_CLASS_STREAMS
#define DB2_CLASS_STREAMS 1
#endif
// Side streams of the calling thread on the current device, for running the
// tile classes of one assembly concurrently (they write disjoint rows).
struct SideStreams {
  static constexpr int kMax = 16;
  cudaStream_t s[kMax] = {};
  cudaEvent_t done[kMax] = {};
  cudaEvent_t fork = nullptr;
  bool ready = false;
};
inline SideStreams& side_streams() {
  thread_local SideStreams per_device[64];
  int dev = 0;
  cudaGetDevice(&dev);
  SideStreams& S = per_device[dev & 63];
  if (!S.ready) {
    for (int i = 0; i < SideStreams::kMax; ++i) {
      cudaStreamCreateWithFlags(&S.s[i], cudaStreamNonBlocking);
      cudaEventCreateWithFlags(&S.done[i], cudaEventDisableTiming);
    }
    cudaEventCreateWithFlags(&S.fork, cudaEventDisableTiming);
    check_cuda("side streams");
    S.ready = true;
  }
  return S;
}

// One launch per shared-memory class.  The classes write disjoint rows, so
// they run on side streams forked from and joined back to the caller's
// stream: the shared-memory-heavy vertex-row tiles (launched first) and the
// register-heavy edge-row tiles then share the SMs instead of each running
// alone below the SM's residency limits.
template <int D, int P, int FORM, bool KP1, int LOADM, typename CT>
void run_assemble(const AsmParams& p, const LaunchCfg& cfg) {
  const int var = (cfg.escapes ? VAR_ESC : 0) | (p.bc_flags ? VAR_BC : 0);
  auto kern = var == 0         ? k_assemble<D, P, FORM, KP1, LOADM, CT, 0>
              : var == VAR_ESC ? k_assemble<D, P, FORM, KP1, LOADM, CT, VAR_ESC>
              : var == VAR_BC  ? k_assemble<D, P, FORM, KP1, LOADM, CT, VAR_BC>
                               : k_assemble<D, P, FORM, KP1, LOADM, CT, VAR_ESC | VAR_BC>;
  static unsigned long long configured[4] = {0, 0, 0, 0};
  allow_dynamic_smem(kern, configured[var]);
  const auto& cb = *cfg.class_begin;
  const int ncls = int(cb.size()) - 1;
  const bool fork = DB2_CLASS_STREAMS && ncls > 1 && ncls <= SideStreams::kMax;
  SideStreams* S = fork ? &side_streams() : nullptr;
  if (fork) cudaEventRecord(S->fork, cfg.stream);
  int used = 0;
  for (int k = ncls - 1; k >= 0; --k) {  // largest segments first
    const int n = cb[k + 1] - cb[k];
    if (n <= 0) continue;
    AsmParams q = p;
    q.tiles = p.tiles + cb[k];
    // the class's row segment (class sizes count doubles; the FP32 path
    // accumulates in floats), one load partial per thread, and 16 bytes of
    // slack for staging the segment at its destination's alignment
    const size_t smem = size_t((*cfg.class_smem)[k]) * sizeof(CT) / sizeof(double) +
                        size_t(cfg.threads) * sizeof(double) + 16;
    cudaStream_t st = cfg.stream;
    if (fork) {
      st = S->s[used];
      cudaStreamWaitEvent(st, S->fork, 0);
    }
    kern<<<n, cfg.threads, smem, st>>>(q);
    count_launch();
    if (fork) cudaEventRecord(S->done[used], st);
    ++used;
  }
  if (fork)
    for (int i = 0; i < used; ++i) cudaStreamWaitEvent(cfg.stream, S->done[i], 0);
  check_cuda("assemble launch");
}

// Dispatch of the load mode / kappa / precision for one (D, P, FORM).
template <int D, int P, int FORM>
bool dispatch(const AsmParams& p, const LaunchCfg& cfg, bool kp1, int loadm, bool fp32) {
#define DB2_RUN(KP1_, LM_)                                                               \
  do {                                                                                   \
    if (fp32) run_assemble<D, P, FORM, KP1_, LM_, float>(p, cfg);                         \
    else run_assemble<D, P, FORM, KP1_, LM_, double>(p, cfg);                             \
    return true;                                                                         \
  } while (0)
  if constexpr (FORM == FORM_ELAS) {
    if (kp1) return false;
    if (loadm == LOAD_NONE) DB2_RUN(false, LOAD_NONE);
    if (loadm == LOAD_CONST) DB2_RUN(false, LOAD_CONST);
    return false;
  } else {
    if (kp1) {
      if (loadm == LOAD_NONE) DB2_RUN(true, LOAD_NONE);
      if (loadm == LOAD_CONST) DB2_RUN(true, LOAD_CONST);
      if (loadm == LOAD_P1) DB2_RUN(true, LOAD_P1);
      if (loadm == LOAD_KP1) DB2_RUN(true, LOAD_KP1);
    } else {
      if (loadm == LOAD_NONE) DB2_RUN(false, LOAD_NONE);
      if (loadm == LOAD_CONST) DB2_RUN(false, LOAD_CONST);
      if (loadm == LOAD_P1) DB2_RUN(false, LOAD_P1);
    }
    return false;
  }
#undef DB2_RUN
}

// Per-translation-unit entry points (assemble_*.cu).
bool dispatch_tet_diff(int P, const AsmParams& p, const LaunchCfg& cfg, bool kp1, int loadm, bool fp32);
bool dispatch_tri_diff(int P, const AsmParams& p, const LaunchCfg& cfg, bool kp1, int loadm, bool fp32);
bool dispatch_tet_elas(int P, const AsmParams& p, const LaunchCfg& cfg, bool kp1, int loadm, bool fp32);

}  // namespace dev
}  // namespace db2
