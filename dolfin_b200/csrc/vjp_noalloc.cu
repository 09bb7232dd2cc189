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
// 524,288 tetrahedra or 699,050 triangles.  Every GPU that loads the library
// holds these 16 MiB until the process exits.
constexpr size_t kNoAllocScratchDoubles = size_t(1) << 21;
static __device__ __align__(256) double g_vjp_scratch[kNoAllocScratchDoubles];

namespace {
std::mutex g_mutex;
constexpr int kMaxDevices = 64;
double* g_scratch_addr[kMaxDevices] = {};

// The device address of g_vjp_scratch on the current device.  In host code
// the array's name is only a host-side stand-in, so the address is looked up
// once per device (with that device current) and cached.
double* scratch_on_current_device() {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) fail(DB2_ERR_CUDA, "cudaGetDevice: %s", cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices) fail(DB2_ERR_UNSUPPORTED, "device index %d", dev);
  std::lock_guard<std::mutex> lock(g_mutex);
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_vjp_scratch);
    if (e != cudaSuccess || !p)
      fail(DB2_ERR_CUDA, "cudaGetSymbolAddress(scratch): %s", cudaGetErrorString(e));
    g_scratch_addr[dev] = static_cast<double*>(p);
  }
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
