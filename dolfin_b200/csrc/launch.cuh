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

template <int D, int P, int FORM, bool KP1, int LOADM, typename CT>
void run_assemble(const AsmParams& p, const LaunchCfg& cfg) {
  auto kern = k_assemble<D, P, FORM, KP1, LOADM, CT>;
  static unsigned long long configured = 0;
  allow_dynamic_smem(kern, configured);
  const auto& cb = *cfg.class_begin;
  for (size_t k = 0; k + 1 < cb.size(); ++k) {
    const int n = cb[k + 1] - cb[k];
    if (n <= 0) continue;
    AsmParams q = p;
    q.tiles = p.tiles + cb[k];
    const size_t smem = size_t((*cfg.class_smem)[k]) + size_t(cfg.threads) * sizeof(double);
    kern<<<n, cfg.threads, smem, cfg.stream>>>(q);
    count_launch();
  }
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
