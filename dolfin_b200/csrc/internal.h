// internal.h -- host-side data structures of the engine (not part of the ABI).
#pragma once

#include <cstdint>
#include <memory>
#include <string>
#include <vector>

#include "../../include/dolfin_b200.h"

namespace db2 {

// Thrown inside the library, converted to a status code at the C boundary.
struct Error {
  int code;
  std::string msg;
};
[[noreturn]] void fail(int code, const char* fmt, ...);

// Device buffer with RAII release (cudaFree); defined in device.cu.
struct DeviceBuffer {
  void* ptr = nullptr;
  size_t bytes = 0;
  DeviceBuffer() = default;
  DeviceBuffer(const DeviceBuffer&) = delete;
  DeviceBuffer& operator=(const DeviceBuffer&) = delete;
  ~DeviceBuffer();
  void alloc(size_t nbytes);
  void upload(const void* host, size_t nbytes);  // alloc + synchronous copy
  template <typename T> T* as() const { return static_cast<T*>(ptr); }
};

// ---- mesh ----------------------------------------------------------------
struct Mesh {
  int tdim = 0;
  int64_t nv = 0, nc = 0;
  std::vector<double> x;         // nv * tdim
  std::vector<uint32_t> cells;   // nc * (tdim+1), sorted per cell
  // edges (computed on demand): numbered in sorted (v0<v1) key order
  bool have_edges = false;
  int64_t ne = 0;
  std::vector<uint32_t> cell_edges;  // nc * nedges(tdim), UFC local edge order
  std::vector<uint32_t> edge_vertices;  // ne * 2, sorted vertex pair of each edge
  // exterior facets (computed on demand), in facet-number order -- sorted
  // vertex key, as TopologyComputation numbers entities: cell << 2 | local
  // facet (facet i of a simplex is opposite its local vertex i)
  bool have_facets = false;
  std::vector<uint32_t> ext_facets;
  // device copies: 4 doubles per vertex (coordinates, then the per-call
  // coefficient values the assembly kernels read with the coordinates)
  DeviceBuffer d_x, d_cells, d_ext_facets, d_partials, d_ext_mask;
  bool on_device = false;
  void ensure_device();      // first GPU use: upload coordinates and cells
  void upload_coordinates();
  void compute_edges();
  void compute_exterior_facets();
};

int nverts(int tdim);
int nedges(int tdim);

// ---- function space ---------------------------------------------------------
struct Space {
  std::shared_ptr<Mesh> mesh;
  int degree = 1, vsize = 1;
  int k = 0;              // nodes (scalar dofs) per cell
  int64_t nnodes = 0;     // scalar global dimension
  std::vector<uint32_t> cell_nodes;  // nc * k (natural node numbering)
  // reorder_dofs_serial = True: node_new[node] = reverse Cuthill-McKee number
  // of a (natural) node; dofs are then bs * node_new[node] + c.  Empty for the
  // natural numbering, where dofs are c * nnodes + node.
  std::vector<int32_t> node_new;
  bool reordered() const { return !node_new.empty(); }
  int64_t dof(int c, int64_t node) const {
    return reordered() ? int64_t(vsize) * node_new[node] + c : int64_t(c) * nnodes + node;
  }
  DeviceBuffer d_cell_nodes;
  DeviceBuffer d_edge_vertices;      // P2: sorted endpoints of each edge node
  bool on_device = false;
  void ensure_device();
  int64_t dim() const { return nnodes * vsize; }
};

// ---- sparsity pattern + row-gather plan -------------------------------------
// Node-level graph (the scalar pattern); the dof-level CSR of a vector space
// is its component expansion: row (c,i) = [c'*nnodes + j for c' in 0..bs-1
// for j in nodecols(i)], rowptr(c,i) = c*bs*nnz_node + bs*node_rowptr[i].
struct Tile {
  int32_t comp;   // test component c of the tile's rows
  int32_t n0, n1; // node range [n0, n1)
  int32_t pad;
};

// Exterior-facet plan of a pattern: each boundary node (row owner) with its
// incidences (exterior facet, facet node) in facet-number order -- the order
// of Assembler::assemble_exterior_facets' facet loop.  Each incidence holds
// the facet's vertex ids relabelled so that the row node is canonical (facet
// vertex 0, or facet edge (0,1)), and the column slots within the node row of
// the facet's nodes in canonical facet order.
struct FacetPlan {
  int kf = 0;                        // nodes per facet
  std::vector<uint32_t> bnode;       // boundary nodes, ascending
  std::vector<uint32_t> binc_ptr;    // bnode.size() + 1
  std::vector<uint32_t> bverts;      // tdim vertex ids per incidence
  std::vector<uint8_t> bslot;        // 8 slots per incidence (kf used)
  DeviceBuffer d_bnode, d_binc_ptr, d_bverts, d_bslot;
};

// CSR of a pattern on a reordered space, in the space's numbering.  The
// kernels assemble in the natural numbering (into library scratch) and
// gather: vals[k] = natural_vals[val_src[k]], b[i] = natural_b[dof_src[i]].
struct ReorderedCSR {
  bool built = false;
  std::vector<int32_t> rowptr, cols, val_src, dof_src;
  DeviceBuffer d_rowptr, d_cols, d_val_src, d_dof_src;
  DeviceBuffer d_vals, d_b, d_flags, d_bcv, d_vec;  // natural-order scratch
};

struct Pattern {
  std::shared_ptr<Space> V;
  bool keep_diagonal = false;
  int bs = 1;
  int64_t nnz_node = 0, nnz = 0, nrows = 0;
  std::vector<int32_t> node_rowptr;  // nnodes + 1
  std::vector<int32_t> node_cols;    // nnz_node
  // row-gather plan: node -> incident (cell, local node) in ascending cell order
  int kp = 0;                        // pos bytes per incidence (k rounded up to 4)
  std::vector<uint32_t> inc_ptr;     // nnodes + 1
  std::vector<uint32_t> inc;         // cell | local_node << 28
  std::vector<uint8_t> pos;          // inc.size() * kp: column slot (within the node row)
                                     // of each node of the relabelled cell
  std::vector<uint32_t> cell_inc;    // nc * k: incidence index of (cell, local node)
  std::vector<Tile> tiles;           // grouped by shared-memory class
  std::vector<int32_t> class_begin;  // tiles[class_begin[k] .. class_begin[k+1]) share
  std::vector<int32_t> class_smem;   //   a launch with class_smem[k] bytes of smem
  int tile_threads = 128;            // CTA size of the tile kernel
  int seg_cap_bytes = 0;             // row-segment cap the tiles were cut with
  // node rows the tile kernel assembles: [row_begin, row_end) (a rank's share
  // of a row-partitioned assembly); row_end < 0 = all rows
  int64_t row_begin = 0, row_end = -1;
  // the caller's value and vector arrays hold the row block alone (a rank's
  // CSR rows of nodes [row_begin, row_end), every component, in global row
  // order; b likewise) instead of the whole CSR / vector
  bool block_storage = false;

  int seg_cap = 0;                   // doubles of shared memory of the largest tile
  // Device incidence records (rs = 8 or 16 bytes, one vector load each):
  // int16 offsets, relative to the row's first fixed vertex, of the other
  // vertices of the relabelled cell, then its k column slots.  Records of
  // each block of 32 consecutive nodes are interleaved (record m of node i at
  // rec_goff[i/32] + i%32 + 32 m) so that a warp's loads are contiguous.
  int rs = 8;
  // records whose offsets did not fit 16 bits (stored as -32768; the kernel
  // then reads the cell's vertices through the incidence word)
  int64_t rec_escapes = 0;
  std::vector<uint32_t> rec_goff;    // per 32-node block: first record index
  DeviceBuffer d_node_rowptr, d_inc_ptr, d_inc, d_rec, d_rec_goff, d_cell_inc, d_tiles, d_rowptr, d_cols;
  // each node's first record again, node-indexed: the row walk's first
  // record load needs no rec_goff lookup before it
  DeviceBuffer d_rec_first;
  // matrix-free action: per-cell element actions (cells x bs x k), grown on
  // first use
  mutable DeviceBuffer d_cellvals;
  bool on_device = false;
  void ensure_device();      // first GPU use: upload the plan, expand the CSR
  // dof-level CSR on the host in the natural numbering (component expansion
  // of the node graph) and in the space's numbering (reordered if it is)
  void csr_host_natural(int32_t* rowptr, int32_t* cols) const;
  void csr_host(int32_t* rowptr, int32_t* cols);
  ReorderedCSR reordered;
  std::unique_ptr<FacetPlan> facets;
  const FacetPlan& facet_plan();     // built and uploaded on first use
};

// Relabelling of a cell so that local node `li` becomes canonical: for a
// vertex node, that vertex first and the others ascending; for an edge node
// (p,q), p and q first.  perm[a] = original local vertex at new position a.
void canonical_perm(int tdim, int li, int perm[4]);
// map[j] = original local node of the relabelled cell's local node j.
void canonical_node_map(int tdim, int degree, int li, int* map);

std::shared_ptr<Mesh> make_unit_cube(int nx, int ny, int nz);
std::shared_ptr<Mesh> make_unit_square(int nx, int ny, int diagonal);
std::shared_ptr<Mesh> make_mesh(int tdim, int64_t nv, const double* x, int64_t nc,
                                const uint32_t* cells);
std::shared_ptr<Space> make_space(std::shared_ptr<Mesh> m, int degree, int vsize);
std::shared_ptr<Pattern> make_pattern(std::shared_ptr<Space> V, bool keep_diagonal,
                                      int tile_threads = 0, int seg_cap_bytes = 0);
// Reordered numbering (reorder_host.cpp): RCM number of each natural node; the
// reordered CSR of a pattern.
std::vector<int32_t> rcm_node_order(const Space& V);
void build_reordered_csr(Pattern& P);
// DOLFIN XML files (io.cpp).
std::shared_ptr<Mesh> read_mesh_xml(const char* path);
void write_mesh_xml(const Mesh& m, const char* path);
std::shared_ptr<Mesh> read_mesh_xdmf(const char* path);
void write_mesh_xdmf(const Mesh& m, const char* path, const double* values, int value_size,
                     const char* name);
void write_vector_xml(const char* path, int64_t n, const double* x);
int64_t read_vector_xml(const char* path, double* x, int64_t cap);  // x NULL: size only
// Host-side facet plan of a pattern (no device work); Pattern::facet_plan()
// also uploads it.
void build_facet_plan(Pattern& P);
// Re-cut the tiles of an existing plan (autotuning), re-uploading d_tiles.
void retile(Pattern& P, int tile_threads, int seg_cap_bytes);
// Tiles of a pattern for a launch shape (pure; does not modify P).
std::vector<Tile> cut_tiles(const Pattern& P, int tile_threads, int seg_cap_doubles, int* max_seg,
                            int64_t node_begin = 0, int64_t node_end = -1);
void set_row_range(Pattern& P, int64_t node_begin, int64_t node_end, bool block_storage = false);
// Where the kernels put CSR value (c, k) and b entry (c, node): see AsmParams.
struct OutputLayout {
  int64_t vstride, vbase, bstride, bbase;
};
OutputLayout output_layout(const Pattern& P);
// Size of a pattern's row block (the whole pattern without a range).
void row_block_size(const Pattern& P, int64_t* nrows, int64_t* nnz);

// Launchers (kernels.cu).  All return after enqueueing on `stream`.
struct FormArgs {
  db2_form f;
  const double* w = nullptr;   // device P1 field or null
};
void launch_assemble(const Pattern& P, const FormArgs* a, const FormArgs* L, int precision,
                     double* vals, double* b, bool add_values, const uint8_t* bc_flags,
                     const double* bc_vals, void* stream);
// Exterior-facet and functional assembly (facets.cu).
void launch_facet_matrix(Pattern& P, const FormArgs& a, double* vals, bool add_values,
                         const uint8_t* bc_flags, const double* bc_vals, double* b, void* stream);
void launch_facet_vector(Pattern& P, const FormArgs& L, double* b, bool add_values,
                         const uint8_t* bc_flags, void* stream);
void launch_functional(Mesh& m, const FormArgs& M, double* out, void* stream);
// Element tensors of listed cells (local.cu).
void launch_local(Space& V, const FormArgs* a, const FormArgs* a_ds, int64_t ncells,
                  const uint32_t* list, double* out, void* stream);
void launch_apply(const Pattern& P, const FormArgs& a, int precision, const double* x, double* y,
                  void* stream);
void launch_vjp(const Pattern& P, const FormArgs& a, const FormArgs& L, int precision,
                const double* gA, const double* gb, double* dkappa, double* scratch,
                void* stream);
void launch_expand_csr(const Pattern& P);
void count_launch(int n = 1);
void check_cuda(const char* what);
size_t vjp_scratch_doubles(const Pattern& P);
// Load the adjoint kernels onto the current device (lazy module loading
// would otherwise do it, allocating, at their first launch).
void preload_vjp_kernels();
// 1 if a tensor-core kernel's bounded wait ran out since the process started
// (its outputs were written as NaN); reads the device flag synchronously.
int tensor_core_status();
// Once per device: set up the allocation-free adjoint's fixed scratch array
// (vjp_noalloc.cu); called by Pattern::ensure_device.
void noalloc_prepare_device();

}  // namespace db2
