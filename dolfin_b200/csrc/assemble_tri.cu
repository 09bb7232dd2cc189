// Instantiations: scalar diffusion (+ load) on triangles, P1 and P2.
#include "launch.cuh"
namespace db2 {
namespace dev {
bool dispatch_tri_diff(int P, const AsmParams& p, const LaunchCfg& cfg, bool kp1, int loadm, bool fp32) {
  if (P == 1) return dispatch<2, 1, FORM_DIFF>(p, cfg, kp1, loadm, fp32);
  if (P == 2) return dispatch<2, 2, FORM_DIFF>(p, cfg, kp1, loadm, fp32);
  return false;
}
}  // namespace dev
}  // namespace db2
