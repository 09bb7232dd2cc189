// device.cu -- device memory helpers, error checks and the CSR expansion kernel.
#include <cuda_runtime.h>

#include <atomic>
#include <cstdio>

#include "internal.h"

namespace db2 {

static std::atomic<int64_t> g_launches{0};
void count_launch(int n) { g_launches += n; }
int64_t launches() { return g_launches.load(); }

void check_cuda(const char* what) {
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) fail(DB2_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

DeviceBuffer::~DeviceBuffer() {
  if (ptr) cudaFree(ptr);
}

void DeviceBuffer::alloc(size_t nbytes) {
  if (ptr) {
    cudaFree(ptr);
    ptr = nullptr;
    bytes = 0;
  }
  if (nbytes == 0) return;
  const cudaError_t e = cudaMalloc(&ptr, nbytes);
  if (e != cudaSuccess) {
    ptr = nullptr;
    cudaGetLastError();
    fail(e == cudaErrorMemoryAllocation ? DB2_ERR_NOMEM : DB2_ERR_CUDA,
         "cudaMalloc(%zu bytes): %s", nbytes, cudaGetErrorString(e));
  }
  bytes = nbytes;
}

void DeviceBuffer::upload(const void* host, size_t nbytes) {
  alloc(nbytes);
  if (nbytes == 0) return;
  const cudaError_t e = cudaMemcpy(ptr, host, nbytes, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) fail(DB2_ERR_CUDA, "cudaMemcpy H2D: %s", cudaGetErrorString(e));
}

// Vertex records of 4 doubles -- (x, y, z, kappa) in 3D, (x, y, kappa, f) in
// 2D -- so that a vertex is one aligned 256-bit load; the coefficient slots
// are written per assembly call (pack_vertex_records).
void Mesh::upload_coordinates() {
  const int w = 4;
  std::vector<double> pad(size_t(nv) * w, 0.0);
  for (int64_t v = 0; v < nv; ++v)
    for (int r = 0; r < tdim; ++r) pad[v * w + r] = x[v * tdim + r];
  d_x.upload(pad.data(), pad.size() * sizeof(double));
}

// Dof-level CSR of a (vector) space from the node-level graph: row (c, i)
// holds the columns e*nnodes + j for every component e and node neighbour j
// -- exactly the rows SparsityPatternBuilder inserts for a component-major
// vector dofmap, already sorted.
__global__ void k_expand_csr(const int32_t* __restrict__ node_rowptr,
                             const int32_t* __restrict__ node_cols, int64_t nnodes,
                             int64_t nnz_node, int bs, int32_t* __restrict__ rowptr,
                             int32_t* __restrict__ cols) {
  const int64_t r = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  const int64_t nrows = nnodes * bs;
  if (r > nrows) return;
  if (r == nrows) {
    rowptr[nrows] = int32_t(nnz_node * bs * bs);
    return;
  }
  const int64_t c = r / nnodes, i = r - c * nnodes;
  const int32_t a = node_rowptr[i], L = node_rowptr[i + 1] - a;
  const int64_t rp = c * bs * nnz_node + int64_t(bs) * a;
  rowptr[r] = int32_t(rp);
  for (int e = 0; e < bs; ++e)
    for (int t = 0; t < L; ++t) cols[rp + int64_t(e) * L + t] = int32_t(e * nnodes + node_cols[a + t]);
}

void launch_expand_csr(const Pattern& P) {
  DeviceBuffer d_ncols;
  d_ncols.upload(P.node_cols.data(), P.node_cols.size() * sizeof(int32_t));
  const_cast<Pattern&>(P).d_rowptr.alloc(size_t(P.nrows + 1) * sizeof(int32_t));
  const_cast<Pattern&>(P).d_cols.alloc(size_t(P.nnz) * sizeof(int32_t));
  const int64_t n = P.nrows + 1;
  const int threads = 256;
  k_expand_csr<<<unsigned((n + threads - 1) / threads), threads>>>(
      P.d_node_rowptr.as<int32_t>(), d_ncols.as<int32_t>(), P.V->nnodes, P.nnz_node, P.bs,
      P.d_rowptr.as<int32_t>(), P.d_cols.as<int32_t>());
  count_launch();
  check_cuda("expand_csr launch");
  const cudaError_t e = cudaDeviceSynchronize();
  if (e != cudaSuccess) fail(DB2_ERR_CUDA, "expand_csr: %s", cudaGetErrorString(e));
}

}  // namespace db2
