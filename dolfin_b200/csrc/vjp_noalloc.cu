// vjp_noalloc.cu -- the adjoint with a fixed, library-owned scratch array.
//
// db2_vjp_kappa keeps its per-cell work array in memory it allocates on
// first use.  Some callers cannot let a library allocate device memory when
// they call it: applications whose device memory is owned by their own pool
// allocator (a cudaMalloc behind the pool's back breaks its accounting and
// can fail once the pool has reserved the device), or loops with streams in
// flight where cudaMalloc's implicit synchronisation would stall them.  For
// those callers db2_vjp_kappa_noalloc uses the static device array below
// instead; it allocates nothing and frees nothing.
#include <cuda_runtime.h>

#include <functional>
#include <mutex>

#include "internal.h"

struct db2_pattern_t;

namespace db2 {
std::shared_ptr<Pattern> pattern_of(db2_pattern P);
int guard_call(const std::function<void()>& f);

// Largest work array the entry point can use: C (d+1) doubles, i.e. up to
// 524,288 tetrahedra or 699,050 triangles.
constexpr size_t kNoAllocScratchDoubles = size_t(1) << 21;
static __device__ __align__(256) double g_vjp_scratch[kNoAllocScratchDoubles];

namespace {
std::mutex g_mutex;
constexpr int kMaxDevices = 64;
double* g_scratch_addr[kMaxDevices] = {};
}  // namespace

// Set-up, once per device, with that device current; called when a pattern
// is first made resident (Pattern::ensure_device), which allocates anyway.
// With lazy module loading (the CUDA 12 default) the 16 MiB array and the
// adjoint kernels reach the device only when first used; looking the array
// up here and loading the kernels here keeps that out of the entry point.
// In host code the array's name is only a host-side stand-in, so its device
// address is looked up (cudaGetSymbolAddress) and cached per device.  From
// then on the device holds the array until the process exits.
void noalloc_prepare_device() {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) fail(DB2_ERR_CUDA, "cudaGetDevice: %s", cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices) return;  // such devices refuse the entry point instead
  std::lock_guard<std::mutex> lock(g_mutex);
  if (g_scratch_addr[dev]) return;
  void* p = nullptr;
  e = cudaGetSymbolAddress(&p, g_vjp_scratch);
  if (e != cudaSuccess || !p)
    fail(DB2_ERR_CUDA, "cudaGetSymbolAddress(scratch): %s", cudaGetErrorString(e));
  preload_vjp_kernels();
  g_scratch_addr[dev] = static_cast<double*>(p);
}

namespace {
// The cached device address of g_vjp_scratch on the current device; never
// looks it up (that could load the module, i.e. allocate).
double* scratch_on_current_device() {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) fail(DB2_ERR_CUDA, "cudaGetDevice: %s", cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices) fail(DB2_ERR_UNSUPPORTED, "device index %d", dev);
  std::lock_guard<std::mutex> lock(g_mutex);
  if (!g_scratch_addr[dev])
    fail(DB2_ERR_ARGUMENT,
         "db2_vjp_kappa_noalloc: no pattern has been made resident on device %d yet (its "
         "fixed scratch array is set up then); assemble with the pattern on this device first",
         dev);
  return g_scratch_addr[dev];
}
}  // namespace
}  // namespace db2

extern "C" int db2_vjp_kappa_noalloc(db2_pattern Ph, const db2_form* a, const double* kappa,
                                     const db2_form* L, const double* f, const double* gA,
                                     const double* gb, int precision, double* dkappa,
                                     void* stream) {
  return db2::guard_call([&] {
    using namespace db2;
    auto P = pattern_of(Ph);
    if (!P || !a || !kappa || !gA || !dkappa) fail(DB2_ERR_ARGUMENT, "NULL argument");
    const size_t need = vjp_scratch_doubles(*P);
    if (need > kNoAllocScratchDoubles)
      fail(DB2_ERR_SHAPE,
           "db2_vjp_kappa_noalloc needs %zu scratch doubles but its fixed array holds %zu "
           "(at most 524288 tetrahedra / 699050 triangles); use db2_vjp_kappa",
           need, kNoAllocScratchDoubles);
    if (P->V->reordered())
      fail(DB2_ERR_UNSUPPORTED,
           "db2_vjp_kappa_noalloc does not take patterns on reordered spaces (their gradients "
           "need library scratch); use db2_vjp_kappa");
    if (P->block_storage)
      fail(DB2_ERR_UNSUPPORTED, "the adjoint takes whole-CSR gradients (no row-block storage)");
    if (!P->on_device)
      fail(DB2_ERR_ARGUMENT,
           "pattern is not resident on the device yet; assemble with it (or call "
           "db2_pattern_csr_device) once before db2_vjp_kappa_noalloc, which allocates nothing");
    double* scratch = scratch_on_current_device();
    FormArgs fa;
    fa.f = *a;
    fa.w = kappa;
    FormArgs fl;
    if (L) {
      fl.f = *L;
      fl.w = f;
    } else {
      fl.f = db2_form{};
      fl.f.kind = DB2_FORM_LOAD;
      fl.f.coeff = DB2_COEFF_NONE;
    }
    // The kernels overwrite every entry they read of the scratch array, so
    // nothing left by an earlier call needs clearing.
    launch_vjp(*P, fa, fl, precision, gA, L ? gb : nullptr, dkappa, scratch, stream);
  });
}
