// batch.cu -- batched multi-mesh assembly: every tile of every member mesh
// in ONE persistent launch, captured once into a CUDA graph.
//
// Members may mix elements (P1/P2, triangles/tetrahedra) but all assemble
// kappa*inner(grad(u), grad(v))*dx with a P1 kappa (the batched workload of
// the benchmark).  Tiles are ordered largest-first (longest-processing-time
// order) and handed out by an atomic counter; each tile's output is produced
// by exactly one CTA with the same arithmetic as the single-mesh kernel, so
// the result is independent of the schedule (bitwise).
#include <cuda_runtime.h>

#include <algorithm>
#include <functional>
#include <numeric>

#include "launch.cuh"

namespace db2 {
dev::AsmParams make_params(const Pattern& P);

namespace dev {

enum { KIND_P1TRI = 0, KIND_P2TRI = 1, KIND_P1TET = 2, KIND_P2TET = 3 };

struct BatchMember {
  AsmParams p;
  int kind;
  int tdim;
  int64_t nv;
  double* xw;
  const double* kappa;
};

struct BatchTile {
  int32_t member;
  int32_t comp;
  int32_t n0, n1;
};

// Members carry no Dirichlet data (their parameters leave bc_flags null), so
// the tiles run the instantiation without boundary-condition state.
template <typename CT>
__device__ __forceinline__ void batch_tile(const BatchMember& m, const Tile& t, double* acc) {
  switch (m.kind) {
    case KIND_P1TRI: tile_body<2, 1, FORM_DIFF, true, LOAD_NONE, CT, 0>(m.p, t, acc); break;
    case KIND_P2TRI: tile_body<2, 2, FORM_DIFF, true, LOAD_NONE, CT, 0>(m.p, t, acc); break;
    case KIND_P1TET: tile_body<3, 1, FORM_DIFF, true, LOAD_NONE, CT, 0>(m.p, t, acc); break;
    default: tile_body<3, 2, FORM_DIFF, true, LOAD_NONE, CT, 0>(m.p, t, acc); break;
  }
}

// Persistent: each CTA repeatedly takes the next tile from the work counter.
// Register cap 64 (16 resident 64-thread CTAs per SM): the batched members
// are 2D meshes, whose rows need fewer registers; measured on B200 for 512
// triangle meshes (ms per graph replay): 0.770 at 64 registers against 0.788
// at 72, 0.847 at 80 (some spills at 64 and 72, none at 96: 0.975); with
// the tiles' Dirichlet-free instantiation (fewer spills) 0.673 at 64 against
// 0.716 at 72.
#ifndef DB2_BATCH_MAXNREG
#define DB2_BATCH_MAXNREG 64
#endif
template <typename CT>
__global__ void __maxnreg__(DB2_BATCH_MAXNREG) k_batch(const BatchMember* __restrict__ members,
                                                           const BatchTile* __restrict__ tiles,
                                                           int ntiles, unsigned int* counter) {
  extern __shared__ __align__(16) double acc[];
  __shared__ int next;
  for (;;) {
    if (threadIdx.x == 0) next = int(atomicAdd(counter, 1u));
    __syncthreads();
    const int t = next;
    __syncthreads();
    if (t >= ntiles) break;
    const BatchTile bt = tiles[t];
    const Tile tile{bt.comp, bt.n0, bt.n1, 0};
    batch_tile<CT>(members[bt.member], tile, acc);
  }
}

// kappa into the w (3D) or third (2D) slot of every member's vertex records.
__global__ void k_batch_pack(const BatchMember* __restrict__ members, int nmembers,
                             const int64_t* __restrict__ vstart, int64_t nvtot) {
  const int64_t g = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (g >= nvtot) return;
  int lo = 0, hi = nmembers;  // member with vstart[m] <= g < vstart[m+1]
  while (hi - lo > 1) {
    const int mid = (lo + hi) / 2;
    if (vstart[mid] <= g) lo = mid;
    else hi = mid;
  }
  const BatchMember& m = members[lo];
  const int64_t v = g - vstart[lo];
  m.xw[4 * v + (m.tdim == 3 ? 3 : 2)] = m.kappa[v];
}

}  // namespace dev

namespace {
struct Batch {
  std::vector<std::shared_ptr<Pattern>> patterns;
  std::vector<dev::BatchMember> members;
  std::vector<dev::BatchTile> tiles;         // LPT order (persistent kernel)
  std::vector<dev::BatchTile> member_tiles;  // member order (reference loop)
  std::vector<int> member_first;             // member_tiles range per member
  std::vector<int64_t> vstart;
  DeviceBuffer d_members, d_tiles, d_member_tiles, d_vstart, d_counter;
  int threads = 128, ctas = 0, smem = 0;
  int64_t cells = 0;
  cudaGraphExec_t exec[2] = {nullptr, nullptr};
  ~Batch() {
    for (auto& e : exec)
      if (e) cudaGraphExecDestroy(e);
  }
};

template <typename CT>
void set_smem_attr() {
  static unsigned long long done = 0;
  dev::allow_dynamic_smem(dev::k_batch<CT>, done);
}

void enqueue_pack(Batch& B, cudaStream_t s) {
  const int64_t nvtot = B.vstart.back();
  dev::k_batch_pack<<<unsigned((nvtot + 255) / 256), 256, 0, s>>>(
      B.d_members.as<dev::BatchMember>(), int(B.members.size()), B.d_vstart.as<int64_t>(), nvtot);
  count_launch();
}

template <typename CT>
void enqueue_persistent(Batch& B, cudaStream_t s) {
  cudaMemsetAsync(B.d_counter.ptr, 0, sizeof(unsigned int), s);
  enqueue_pack(B, s);
  dev::k_batch<CT><<<B.ctas, B.threads, size_t(B.smem), s>>>(
      B.d_members.as<dev::BatchMember>(), B.d_tiles.as<dev::BatchTile>(), int(B.tiles.size()),
      B.d_counter.as<unsigned int>());
  count_launch();
}

// The reference loop: one launch per member over that member's tiles.  It
// runs the same k_batch kernel as the persistent path (with the member's tile
// range and a counter of its own): two kernels that each inline tile_body may
// be compiled with different multiply-add fusion, and the loop is the check
// that the persistent schedule does not change a single bit.
template <typename CT>
void enqueue_loop(Batch& B, cudaStream_t s) {
  // the vertex-record pack covers all members at once (a slice of it is not
  // separable), then one launch per member
  const size_t nm = B.members.size();
  cudaMemsetAsync(B.d_counter.ptr, 0, (nm + 1) * sizeof(unsigned int), s);
  enqueue_pack(B, s);
  for (size_t m = 0; m < nm; ++m) {
    const int t0 = B.member_first[m], n = B.member_first[m + 1] - t0;
    if (n <= 0) continue;
    dev::k_batch<CT><<<std::min(n, B.ctas), B.threads, size_t(B.smem), s>>>(
        B.d_members.as<dev::BatchMember>(), B.d_member_tiles.as<dev::BatchTile>() + t0, n,
        B.d_counter.as<unsigned int>() + 1 + m);
    count_launch();
  }
}
}  // namespace

}  // namespace db2

struct db2_batch_t {
  db2::Batch B;
};
struct db2_pattern_t;
namespace db2 {
std::shared_ptr<Pattern> pattern_of(db2_pattern P);
int guard_call(const std::function<void()>& f);
}

extern "C" {

int db2_batch_create(int count, const db2_pattern* patterns, const db2_form* forms,
                     const double* const* kappas, double* const* vals, int tile_threads,
                     int seg_cap_bytes, int ctas_per_sm, db2_batch* out) {
  return db2::guard_call([&] {
    using namespace db2;
    if (count <= 0 || !patterns || !forms || !kappas || !vals || !out)
      fail(DB2_ERR_ARGUMENT, "batch: empty or NULL arguments");
    const int threads = tile_threads > 0 ? tile_threads : 128;
    if (threads % 32 || threads > dev::kMaxTileThreads) fail(DB2_ERR_ARGUMENT, "batch: tile_threads");
    const int cap = seg_cap_bytes > 0 ? seg_cap_bytes : 24 * 1024;
    auto* h = new db2_batch_t;
    Batch& B = h->B;
    try {
      B.threads = threads;
      B.vstart.push_back(0);
      int max_seg = 0;
      B.member_first.push_back(0);
      for (int m = 0; m < count; ++m) {
        auto P = pattern_of(patterns[m]);
        if (!P) fail(DB2_ERR_ARGUMENT, "batch member %d: NULL pattern", m);
        if (P->V->reordered()) fail(DB2_ERR_UNSUPPORTED, "batch member %d: reordered space", m);
        if (forms[m].kind != DB2_FORM_DIFFUSION || forms[m].coeff != DB2_COEFF_P1 || P->bs != 1)
          fail(DB2_ERR_UNSUPPORTED, "batch member %d: only kappa*grad.grad with a P1 kappa", m);
        if (!kappas[m] || !vals[m]) fail(DB2_ERR_ARGUMENT, "batch member %d: NULL kappa/vals", m);
        if (reinterpret_cast<uintptr_t>(vals[m]) % alignof(double))
          fail(DB2_ERR_ARGUMENT, "batch member %d: vals must be 8-byte aligned", m);
        P->ensure_device();
        if (P->rec_escapes)
          fail(DB2_ERR_UNSUPPORTED,
               "batch member %d: cell vertex ids more than 32767 apart (assemble it on its own, "
               "which handles any numbering)", m);
        B.patterns.push_back(P);
        dev::BatchMember bm{};
        bm.p = make_params(*P);
        bm.p.kappa = kappas[m];
        bm.p.kscale = 1.0;
        bm.p.vals = vals[m];
        const int D = P->V->mesh->tdim, deg = P->V->degree;
        bm.kind = D == 2 ? (deg == 1 ? dev::KIND_P1TRI : dev::KIND_P2TRI)
                         : (deg == 1 ? dev::KIND_P1TET : dev::KIND_P2TET);
        bm.tdim = D;
        bm.nv = P->V->mesh->nv;
        bm.xw = P->V->mesh->d_x.as<double>();
        bm.kappa = kappas[m];
        B.members.push_back(bm);
        B.vstart.push_back(B.vstart.back() + bm.nv);
        B.cells += P->V->mesh->nc;
        int ms = 0;
        for (const Tile& t : cut_tiles(*P, threads, cap / 8, &ms))
          B.member_tiles.push_back(dev::BatchTile{m, t.comp, t.n0, t.n1});
        B.member_first.push_back(int(B.member_tiles.size()));
        max_seg = std::max(max_seg, ms);
      }
      // largest tiles first (work ~ incidences of the tile)
      B.tiles = B.member_tiles;
      auto work = [&](const dev::BatchTile& t) {
        const auto& P = *B.patterns[t.member];
        return int64_t(P.inc_ptr[t.n1]) - int64_t(P.inc_ptr[t.n0]);
      };
      std::stable_sort(B.tiles.begin(), B.tiles.end(),
                       [&](const dev::BatchTile& a, const dev::BatchTile& b) { return work(a) > work(b); });
      B.smem = max_seg * 8 + B.threads * 8 + 16;  // + alignment slack of tile_body
      int dev_id = 0, nsm = 0;
      cudaGetDevice(&dev_id);
      cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev_id);
      set_smem_attr<double>();
      set_smem_attr<float>();
      int occ = 0;
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, dev::k_batch<double>, B.threads, size_t(B.smem));
      const int per_sm = ctas_per_sm > 0 ? std::min(ctas_per_sm, std::max(occ, 1)) : std::max(occ, 1);
      B.ctas = nsm * per_sm;
      B.d_members.upload(B.members.data(), B.members.size() * sizeof(dev::BatchMember));
      B.d_tiles.upload(B.tiles.data(), B.tiles.size() * sizeof(dev::BatchTile));
      B.d_member_tiles.upload(B.member_tiles.data(), B.member_tiles.size() * sizeof(dev::BatchTile));
      B.d_vstart.upload(B.vstart.data(), B.vstart.size() * sizeof(int64_t));
      B.d_counter.alloc((B.members.size() + 1) * sizeof(unsigned int));
      check_cuda("batch create");
    } catch (...) {
      delete h;
      throw;
    }
    *out = h;
  });
}

int db2_batch_info(db2_batch B, int64_t* tiles, int64_t* cells, int* ctas) {
  return db2::guard_call([&] {
    if (!B) db2::fail(DB2_ERR_ARGUMENT, "batch is NULL");
    if (tiles) *tiles = int64_t(B->B.tiles.size());
    if (cells) *cells = B->B.cells;
    if (ctas) *ctas = B->B.ctas;
  });
}

// The persistent launch (counter reset, kappa packing, assembly) is captured
// into a CUDA graph on first use per precision and replayed on `stream`.
int db2_batch_assemble(db2_batch Bh, int precision, void* stream) {
  return db2::guard_call([&] {
    using namespace db2;
    if (!Bh) fail(DB2_ERR_ARGUMENT, "batch is NULL");
    if (precision != DB2_FP64 && precision != DB2_FP32_CONTRACT) fail(DB2_ERR_ARGUMENT, "precision");
    Batch& B = Bh->B;
    cudaGraphExec_t& ex = B.exec[precision];
    if (!ex) {
      cudaStream_t cs;
      if (cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking) != cudaSuccess) check_cuda("batch stream");
      cudaGraph_t g = nullptr;
      cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
      if (precision == DB2_FP64) enqueue_persistent<double>(B, cs);
      else enqueue_persistent<float>(B, cs);
      const cudaError_t e1 = cudaStreamEndCapture(cs, &g);
      cudaStreamDestroy(cs);
      if (e1 != cudaSuccess) fail(DB2_ERR_CUDA, "batch graph capture: %s", cudaGetErrorString(e1));
      const cudaError_t e2 = cudaGraphInstantiate(&ex, g, 0);
      cudaGraphDestroy(g);
      if (e2 != cudaSuccess) {
        ex = nullptr;
        fail(DB2_ERR_CUDA, "batch graph instantiate: %s", cudaGetErrorString(e2));
      }
    }
    const cudaError_t e = cudaGraphLaunch(ex, static_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) fail(DB2_ERR_CUDA, "batch graph launch: %s", cudaGetErrorString(e));
    count_launch(2);
  });
}

int db2_batch_assemble_loop(db2_batch Bh, int precision, void* stream) {
  return db2::guard_call([&] {
    using namespace db2;
    if (!Bh) fail(DB2_ERR_ARGUMENT, "batch is NULL");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (precision == DB2_FP64) enqueue_loop<double>(Bh->B, s);
    else if (precision == DB2_FP32_CONTRACT) enqueue_loop<float>(Bh->B, s);
    else fail(DB2_ERR_ARGUMENT, "precision");
    check_cuda("batch loop launch");
  });
}

int db2_batch_destroy(db2_batch B) {
  delete B;
  return DB2_OK;
}

}  // extern "C"
