// reorder.cu -- device side of the reordered numbering: the kernels assemble
// in the natural numbering into library scratch, then these gathers move the
// result into the caller's arrays in the space's (reordered) numbering, and
// the scatters move reordered inputs (Dirichlet flags/values, vectors,
// upstream gradients) into natural order.  One extra pass over the values:
// 8 B read + 4 B index + 8 B write per nonzero.
#include <cuda_runtime.h>

#include "internal.h"

namespace db2 {
namespace dev {

template <typename T>
__global__ void __launch_bounds__(256) k_gather(T* __restrict__ dst, const T* __restrict__ src,
                                                const int32_t* __restrict__ idx, int64_t n,
                                                int add) {
  const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const T v = src[__ldg(idx + i)];
  dst[i] = add ? T(dst[i] + v) : v;
}

template <typename T>
__global__ void __launch_bounds__(256) k_scatter(T* __restrict__ dst, const T* __restrict__ src,
                                                 const int32_t* __restrict__ idx, int64_t n) {
  const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  dst[__ldg(idx + i)] = src[i];
}

}  // namespace dev

namespace {
unsigned blocks(int64_t n) { return unsigned((n + 255) / 256); }
}  // namespace

ReorderedCSR& reordered_on_device(Pattern& P) {
  ReorderedCSR& R = P.reordered;
  if (!R.built) build_reordered_csr(P);
  if (!R.d_val_src.ptr) {
    R.d_rowptr.upload(R.rowptr.data(), R.rowptr.size() * sizeof(int32_t));
    R.d_cols.upload(R.cols.data(), R.cols.size() * sizeof(int32_t));
    R.d_val_src.upload(R.val_src.data(), R.val_src.size() * sizeof(int32_t));
    R.d_dof_src.upload(R.dof_src.data(), R.dof_src.size() * sizeof(int32_t));
  }
  const int64_t N = P.V->dim();
  if (!R.d_vals.ptr) R.d_vals.alloc(size_t(P.nnz) * sizeof(double));
  if (!R.d_b.ptr) R.d_b.alloc(size_t(N) * sizeof(double));
  if (!R.d_vec.ptr) R.d_vec.alloc(size_t(N) * sizeof(double));
  if (!R.d_flags.ptr) R.d_flags.alloc(size_t(N));
  if (!R.d_bcv.ptr) R.d_bcv.alloc(size_t(N) * sizeof(double));
  return R;
}

void gather_values(Pattern& P, double* vals, bool add, void* stream) {
  ReorderedCSR& R = reordered_on_device(P);
  dev::k_gather<double><<<blocks(P.nnz), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      vals, R.d_vals.as<double>(), R.d_val_src.as<int32_t>(), P.nnz, add ? 1 : 0);
  count_launch();
  check_cuda("reorder gather launch");
}

void gather_dofs(Pattern& P, double* dst, const double* src_nat, bool add, void* stream) {
  ReorderedCSR& R = reordered_on_device(P);
  const int64_t N = P.V->dim();
  dev::k_gather<double><<<blocks(N), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      dst, src_nat, R.d_dof_src.as<int32_t>(), N, add ? 1 : 0);
  count_launch();
  check_cuda("reorder gather launch");
}

void scatter_dofs(Pattern& P, double* dst_nat, const double* src, void* stream) {
  ReorderedCSR& R = reordered_on_device(P);
  const int64_t N = P.V->dim();
  dev::k_scatter<double><<<blocks(N), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      dst_nat, src, R.d_dof_src.as<int32_t>(), N);
  count_launch();
  check_cuda("reorder scatter launch");
}

void scatter_flags(Pattern& P, uint8_t* dst_nat, const uint8_t* src, void* stream) {
  ReorderedCSR& R = reordered_on_device(P);
  const int64_t N = P.V->dim();
  dev::k_scatter<uint8_t><<<blocks(N), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      dst_nat, src, R.d_dof_src.as<int32_t>(), N);
  count_launch();
  check_cuda("reorder scatter launch");
}

void scatter_values(Pattern& P, double* dst_nat, const double* src, void* stream) {
  ReorderedCSR& R = reordered_on_device(P);
  dev::k_scatter<double><<<blocks(P.nnz), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      dst_nat, src, R.d_val_src.as<int32_t>(), P.nnz);
  count_launch();
  check_cuda("reorder scatter launch");
}

}  // namespace db2
