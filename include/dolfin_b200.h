/*
 * dolfin_b200.h -- C ABI of the B200 finite-element assembly engine.
 *
 * The engine replaces the hot path of DOLFIN 2019.1 assembly
 * (dolfin::Assembler / SystemAssembler and Python dolfin.assemble) for the
 * named Lagrange forms on simplices.  Host structures (mesh, dofmap,
 * sparsity pattern) are built on the CPU exactly as DOLFIN builds them with
 * parameters["reorder_dofs_serial"] = False and uploaded once; assembly runs
 * as hand-written sm_100a kernels on caller-provided device buffers.
 *
 * Conventions
 *   - every entry point returns DB2_OK (0) or a DB2_ERR_* code; the message
 *     of the last failure on the calling thread is db2_last_error().  This
 *     replaces dolfin_error() (dolfin/log/log.cpp:129), which throws.
 *   - pointers documented as "device" are CUDA global-memory pointers on the
 *     current device; "host" pointers are ordinary CPU memory.
 *   - `stream` is a cudaStream_t passed as void* (NULL = legacy default
 *     stream); all device work of a call is ordered on it and the call does
 *     not synchronise unless stated.
 *   - objects are owned by the caller and released with *_destroy; a space
 *     keeps its mesh alive and a pattern keeps its space alive by reference
 *     (destroy in reverse order of creation).
 */
#ifndef DOLFIN_B200_H
#define DOLFIN_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ----------------------------------------------------- */
#define DB2_OK 0
#define DB2_ERR_ARGUMENT 1    /* NULL or out-of-range argument               */
#define DB2_ERR_SHAPE 2       /* dimensions do not match the form/space      */
#define DB2_ERR_INDEX 3       /* vertex/dof index out of range               */
#define DB2_ERR_MESH 4        /* mesh not ordered / degenerate cell          */
#define DB2_ERR_UNSUPPORTED 5 /* element/form combination not provided       */
#define DB2_ERR_CUDA 6        /* CUDA runtime error                          */
#define DB2_ERR_NOMEM 7       /* host or device allocation failed            */
#define DB2_ERR_TIMEOUT 8     /* bounded device wait ran out                 */

/* ---- opaque handles --------------------------------------------------- */
typedef struct db2_mesh_t* db2_mesh;
typedef struct db2_space_t* db2_space;
typedef struct db2_pattern_t* db2_pattern;
typedef struct db2_batch_t* db2_batch;

/* ---- forms ------------------------------------------------------------ */
enum db2_form_kind {
  DB2_FORM_DIFFUSION = 1,  /* a = kappa*inner(grad(u), grad(v))*dx          */
  DB2_FORM_LOAD = 2,       /* L = f*v*dx (scalar), inner(f, v)*dx (vector)  */
  DB2_FORM_ELASTICITY = 3, /* a = inner(sigma(u), epsilon(v))*dx,
                              sigma = 2 mu epsilon + lmbda tr(epsilon) I    */
  /* exterior facet integrals (Assembler::assemble_exterior_facets,
     dolfin/fem/Assembler.cpp:196-288) and functionals                      */
  DB2_FORM_FACET_MASS = 4, /* a = w*u*v*ds (scalar spaces)                  */
  DB2_FORM_FACET_LOAD = 5, /* L = w*v*ds (scalar), inner(t, v)*ds (vector,
                              t = constant[0..2])                           */
  DB2_FORM_FUNCTIONAL = 6, /* M = w*dx                                      */
  DB2_FORM_FACET_FUNCTIONAL = 7 /* M = w*ds                                 */
};
enum db2_coeff_kind {
  DB2_COEFF_NONE = 0,      /* coefficient 1                                 */
  DB2_COEFF_CONSTANT = 1,  /* dolfin Constant: constant[] (scalar or vector)*/
  DB2_COEFF_P1 = 2,        /* P1 Function: device array of vertex values     */
  DB2_COEFF_P1_SCALED = 3, /* constant[0] * P1 Function                      */
  DB2_COEFF_COORD = 4,     /* constant[0] * x[i], i = (int)constant[1]
                              (SpatialCoordinate; functionals only)         */
  DB2_COEFF_P1_KAPPA = 5   /* L = constant[0] * kappa * f * v * dx: f the
                              load's P1 field, kappa the bilinear form's P1
                              field (system assembly of kappa*grad.grad)    */
};
enum db2_precision {
  DB2_FP64 = 0,            /* geometry, contraction, accumulation in FP64    */
  DB2_FP32_CONTRACT = 1,   /* FP64 geometry and global accumulation; the
                              reference-tensor contraction in FP32           */
  DB2_FP32_TENSOR_CORE = 2 /* db2_apply only, P2 tetrahedra, kappa*grad.grad:
                              the FP32 contraction on the tensor cores      */
};

typedef struct {
  int kind;            /* db2_form_kind                                     */
  int coeff;           /* db2_coeff_kind of kappa (a) or f (L)              */
  double constant[3];  /* constant value(s)                                 */
  double mu, lmbda;    /* elasticity Lame constants                         */
} db2_form;

/* ---- library ---------------------------------------------------------- */
const char* db2_last_error(void);
const char* db2_version(void);
/* Number of engine kernels launched by this process so far (all streams). */
int64_t db2_kernel_launches(void);

/* ---- mesh (dolfin::Mesh, dolfin/mesh/Mesh.h; MeshGeometry/MeshTopology) */
/* Mesh from host arrays: coords[nv*tdim] (gdim == tdim), cells[nc*(tdim+1)].
   Each cell's vertex list must be sorted ascending (an ordered mesh,
   DofMapBuilder.cpp:62-68 rejects unordered meshes); replaces
   MeshEditor::open/add_vertex/add_cell/close (dolfin/mesh/MeshEditor.h). */
int db2_mesh_create(int tdim, int64_t nv, const double* coords, int64_t nc,
                    const uint32_t* cells, db2_mesh* out);
/* UnitCubeMesh(nx,ny,nz): BoxMesh::build_tet (dolfin/generation/BoxMesh.cpp:50-170). */
int db2_mesh_unit_cube(int nx, int ny, int nz, db2_mesh* out);
/* UnitSquareMesh(nx,ny,diagonal): RectangleMesh::build_tri
   (dolfin/generation/RectangleMesh.cpp:46-233); diagonal 0 "right", 1 "left",
   2 "right/left", 3 "left/right". */
int db2_mesh_unit_square(int nx, int ny, int diagonal, db2_mesh* out);
int db2_mesh_info(db2_mesh m, int* tdim, int64_t* nv, int64_t* nc);
/* Host copies of Mesh::coordinates() and Mesh::cells(). */
int db2_mesh_copy(db2_mesh m, double* coords, uint32_t* cells);
/* Overwrite vertex coordinates (host array nv*tdim); topology unchanged. */
int db2_mesh_set_coordinates(db2_mesh m, const double* coords);
/* Number of edges (mesh.init(1); TopologyComputation key matching). */
int db2_mesh_num_edges(db2_mesh m, int64_t* ne);
/* Exterior facets (Facet::exterior(): one incident cell), in facet-number
   order (sorted vertex key, TopologyComputation key matching): count, and
   host copies of each facet's cell and local facet index (facet i of a
   simplex is opposite local vertex i). */
int db2_mesh_num_exterior_facets(db2_mesh m, int64_t* n);
int db2_mesh_exterior_facets(db2_mesh m, uint32_t* cell, int32_t* local_facet);
int db2_mesh_destroy(db2_mesh m);

/* ---- files (DOLFIN XML; dolfin/io/XMLMesh.cpp, XMLVector.cpp) -------- */
/* Mesh(filename) / File(filename) >> mesh for a triangle or tetrahedron
   mesh (dim == tdim); cell vertex lists are sorted, as MeshEditor::close
   orders a freshly read mesh. */
int db2_mesh_read_xml(const char* path, db2_mesh* out);
/* File(filename) << mesh. */
int db2_mesh_write_xml(db2_mesh m, const char* path);
/* XDMFFile(path).read(mesh) / .write(mesh) with Encoding.ASCII
   (dolfin/io/XDMFFile.cpp:91-131, 1140-1930): Topology/Geometry DataItems
   inline (Format="XML"); HDF5-backed files are rejected (no HDF5 in this
   build).  Cell vertex lists are sorted on reading.  With values != NULL
   (host, nv x value_size, value_size 1 or tdim) a vertex field named `name`
   is written as a node-centred Attribute, as XDMFFile::write(Function)
   does for a P1 function (:311-397). */
int db2_mesh_read_xdmf(const char* path, db2_mesh* out);
int db2_mesh_write_xdmf(db2_mesh m, const char* path, const double* values, int value_size,
                        const char* name);
/* File(filename) << vector / >> vector for a host array x[n]; read with
   x = NULL returns the size in *n, else reads at most *n values. */
int db2_vector_write_xml(const char* path, int64_t n, const double* x);
int db2_vector_read_xml(const char* path, int64_t* n, double* x);

/* ---- function space + dofmap (DofMap, DofMapBuilder::build) ----------- */
/* Continuous Lagrange P1/P2 with value_size 1 or tdim; natural UFC
   numbering (DofMapBuilder.cpp:253-272), vector spaces component-major. */
int db2_space_create(db2_mesh m, int degree, int value_size, db2_space* out);
/* The same space with the reordered numbering of reorder_dofs_serial = True
   and dof_ordering_library = "Boost" (DofMapBuilder.cpp:168-252,
   compute_node_reordering :1473-1667, BoostGraphOrdering.cpp:34-75): nodes
   numbered by reverse Cuthill-McKee of the node graph, dofs bs*node + c.
   Matrices, vectors, Dirichlet arrays and gradients passed with a pattern
   of this space are in this numbering (the engine assembles in the natural
   numbering into library scratch -- nnz + 3 N doubles -- and gathers);
   coefficient fields stay vertex-indexed. */
int db2_space_create_reordered(db2_mesh m, int degree, int value_size, db2_space* out);
/* node_new[nnodes]: the number of each natural node (identity unless
   reordered); natural node = vertex index, then nv + edge index. */
int db2_space_node_numbers(db2_space V, int32_t* node_new);
int db2_space_info(db2_space V, int* ndofs_per_cell, int64_t* dim);
/* DofMap::cell_dofs for all cells (dolfin/fem/DofMap.h:201-206), host out[nc*ndofs]. */
int db2_space_cell_dofs(db2_space V, int32_t* out);
int db2_space_destroy(db2_space V);

/* ---- sparsity pattern + assembly plan --------------------------------- */
/* SparsityPatternBuilder::build (dolfin/fem/SparsityPatternBuilder.cpp:42-269)
   + EigenMatrix::init (dolfin/la/EigenMatrix.cpp:384-410) for a on V x V:
   sorted CSR (int32 rowptr/cols, as Eigen::SparseMatrix<double,RowMajor,int>),
   plus the engine's row-gather plan.  keep_diagonal as AssemblerBase.h:67.
   Limits of the plan (DB2_ERR_UNSUPPORTED beyond them): fewer than 2^28
   cells (an incidence word holds the cell in 28 bits), at most 255 distinct
   nodes in a node's row (column slots are bytes), nnz and the global
   dimension within int32 (Eigen's StorageIndex).  Any vertex numbering is
   accepted: incidences whose cell spans more than 32767 vertex ids (16-bit
   offsets in the plan's records) read their cell's vertex list instead,
   which costs two dependent loads on those incidences only. */
int db2_pattern_create(db2_space V, int keep_diagonal, db2_pattern* out);
int db2_pattern_info(db2_pattern P, int64_t* nrows, int64_t* nnz);
/* Device CSR arrays owned by the pattern (EigenMatrix::data(),
   dolfin/la/EigenMatrix.h:193-194). */
int db2_pattern_csr_device(db2_pattern P, const int32_t** rowptr, const int32_t** cols);
/* Host copies: rowptr[nrows+1], cols[nnz]. */
int db2_pattern_csr_host(db2_pattern P, int32_t* rowptr, int32_t* cols);
int db2_pattern_destroy(db2_pattern P);
/* Diagnostics of the row-gather plan (no reference counterpart; used by the
   tests and the autotuner): node-level graph, node -> (cell | local node<<28)
   incidences in cell order, per-incidence column slots (kp bytes each), and
   tiles as int32 quadruples (component, first node, end node, 0). */
int db2_pattern_plan_info(db2_pattern P, int64_t* nnodes, int64_t* nincidences, int* kp,
                          int64_t* ntiles, int64_t* ngroups, int64_t* ntypes);
int db2_pattern_plan_copy(db2_pattern P, int32_t* node_rowptr, int32_t* node_cols,
                          uint32_t* inc_ptr, uint32_t* inc, uint8_t* pos, int32_t* tiles);
/* Diagnostics of the exterior-facet plan (no reference counterpart; used by
   the tests): boundary nodes, their (exterior facet, facet node) incidences
   in facet-number order (binc_ptr[nbnodes+1]), per incidence the facet's
   tdim vertex ids relabelled so the row node is canonical (bverts) and the
   CSR column slots of its kf facet nodes within the node's row (bslot, 8
   bytes per incidence). */
int db2_pattern_facet_plan_info(db2_pattern P, int64_t* nbnodes, int64_t* nincidences, int* kf);
int db2_pattern_facet_plan_copy(db2_pattern P, uint32_t* bnode, uint32_t* binc_ptr,
                                uint32_t* bverts, uint8_t* bslot);
/* Re-cut the pattern's tiles (launch shape of the assembly kernel): CTAs of
   tile_threads threads, row segments of at most seg_cap_bytes of shared
   memory.  Results do not depend on the launch shape (bitwise). */
int db2_pattern_retile(db2_pattern P, int tile_threads, int seg_cap_bytes);
/* Row-partitioned assembly (one rank's share of a single mesh): from now on
   the assembly entry points (db2_assemble_matrix, _vector, _system,
   _system_bc, _facets_bc; cell and exterior-facet terms alike) compute and
   write -- or zero, where add_values = 0 -- only the CSR rows and b entries
   of nodes
   [node_begin, node_end), every component, each from all cells around it,
   so no exchange between ranks is needed -- the counterpart of the owned
   row range of DOLFIN's distributed SparsityPattern
   (dolfin/la/SparsityPattern.cpp:200-255, SparsityPattern::apply :441),
   whose off-process entries this design never produces.  Other rows are left
   as they were.  [0, nnodes) restores full assembly.  Natural numbering
   only. */
int db2_pattern_set_row_range(db2_pattern P, int64_t node_begin, int64_t node_end);
/* As db2_pattern_set_row_range, and the value and vector arrays the
   assembly entry points take then hold the row block alone: the CSR rows of
   nodes [node_begin, node_end) of every component, in global row order
   (component-major), and their b entries likewise -- the rows a rank owns in
   DOLFIN's distributed SparsityPattern (dolfin/la/SparsityPattern.cpp:
   200-255), stored without the rest of the matrix.  Sizes:
   db2_pattern_row_block_info; the block's row pointers (from 0) and global
   column indices: db2_pattern_row_block_csr_host.  The adjoint entry points
   refuse row-block storage (their gradients are whole-CSR arrays); the
   matrix-free action is unaffected (x and y stay whole vectors).  The plan
   (incidence records) stays whole on the device. */
int db2_pattern_set_row_block(db2_pattern P, int64_t node_begin, int64_t node_end);
int db2_pattern_row_block_info(db2_pattern P, int64_t* nrows, int64_t* nnz);
int db2_pattern_row_block_csr_host(db2_pattern P, int32_t* rowptr, int32_t* cols);

/* ---- assembly --------------------------------------------------------- */
/* Assembler::assemble(A, a) (dolfin/fem/Assembler.cpp:52-103) for a bilinear
   form on the pattern's space: writes CSR values vals[nnz] (device, 8-byte
   aligned like every double array here; other pointers are refused with
   DB2_ERR_ARGUMENT).  w is
   the device P1 coefficient (kappa) when a.coeff is P1/P1_SCALED.
   add_values as AssemblerBase.h:46 (accumulate into vals). */
int db2_assemble_matrix(db2_pattern P, const db2_form* a, const double* w, int precision,
                        double* vals, int add_values, void* stream);
/* Assembler::assemble(b, L) for a linear form: b[N] (device). */
int db2_assemble_vector(db2_pattern P, const db2_form* L, const double* w, double* b,
                        int add_values, void* stream);
/* db2_assemble_matrix / db2_assemble_vector also take DB2_FORM_FACET_MASS /
   DB2_FORM_FACET_LOAD: the exterior-facet loop of Assembler::assemble
   (Assembler.cpp:196-288).  A form with dx and ds terms is assembled by the
   cell call, then the facet call with add_values = 1 (the reference's cell
   loop, then facet loop). */

/* double assemble(const Form&) (dolfin/fem/assemble.h:66) for
   M = w*dx (DB2_FORM_FUNCTIONAL) or w*ds (DB2_FORM_FACET_FUNCTIONAL), w =
   1, Constant, P1 Function (w: device vertex values) or x[i]
   (DB2_COEFF_COORD): writes the value to out[0] (device).  Deterministic:
   a fixed-order reduction. */
int db2_assemble_scalar(db2_mesh m, const db2_form* M, const double* w, double* out,
                        void* stream);
/* SystemAssembler(a, L).assemble(A, b) (dolfin/fem/SystemAssembler.cpp:138-301,
   cell_wise_assembly :303-492) without boundary conditions: A and b in one
   pass sharing the geometry of each cell. */
int db2_assemble_system(db2_pattern P, const db2_form* a, const double* wa, const db2_form* L,
                        const double* wL, int precision, double* vals, double* b, void* stream);
/* SystemAssembler with DirichletBC: symmetric modification
   SystemAssembler::apply_bc (dolfin/fem/SystemAssembler.cpp:1037-1070) in the
   element epilogue.  bc_flags[N] (device, uint8: 1 = Dirichlet dof) and
   bc_vals[N] (device). */
int db2_assemble_system_bc(db2_pattern P, const db2_form* a, const double* wa, const db2_form* L,
                           const double* wL, const uint8_t* bc_flags, const double* bc_vals,
                           int precision, double* vals, double* b, void* stream);
/* assemble_local (LocalAssembler::assemble, dolfin/fem/LocalAssembler.cpp:
   39-98) for a list of cells: the dense tensor of each cell in its local
   dof order (DofMap::cell_dofs order; vector spaces component-major),
   row-major over (test, trial): out[ncells*n*n] (bilinear) or out[ncells*n]
   (linear), n = dofs per cell, device.  a: the cell integral (diffusion,
   elasticity or load) and/or a_ds: the exterior-facet integral, added for
   the facets of each cell that lie on the boundary.  cells: device
   uint32[ncells]; an index beyond the mesh leaves its tensor unwritten. */
int db2_assemble_local(db2_space V, const db2_form* a, const double* w, const db2_form* a_ds,
                       const double* w_ds, int64_t ncells, const uint32_t* cells, double* out,
                       void* stream);
/* The exterior-facet terms of a SystemAssembler pass with DirichletBC
   (SystemAssembler.cpp:417-470 adds them to the cell tensor before
   apply_bc): call after db2_assemble_system_bc with the same bc_flags /
   bc_vals.  a_ds (DB2_FORM_FACET_MASS) or L_ds (DB2_FORM_FACET_LOAD) may be
   NULL; Dirichlet rows take nothing, Dirichlet columns move to b. */
int db2_assemble_facets_bc(db2_pattern P, const db2_form* a_ds, const double* wa,
                           const db2_form* L_ds, const double* wL, const uint8_t* bc_flags,
                           const double* bc_vals, double* vals, double* b, void* stream);
/* Matrix-free action y = A(a) x (device x[N], y[N]); replaces assembling A
   and calling GenericMatrix::mult (dolfin/la/GenericMatrix.h).  Computed
   per cell (element actions, exact quadrature) and summed per row in cell
   order, so repeated calls agree bitwise.  The first call on a pattern
   allocates cells * bs * k doubles of device work space, kept by the
   pattern; calls on one pattern that overlap on the GPU race on it. */
int db2_apply(db2_pattern P, const db2_form* a, const double* w, int precision, const double* x,
              double* y, void* stream);
/* db2_apply with DB2_FP32_CONTRACT computes the element actions in FP32
   from the FP64 geometry and keeps them in FP32 until the FP64 row sums.
   With DB2_FP32_TENSOR_CORE (P2 tetrahedra, kappa*grad.grad, kappa 1,
   Constant or P1; other forms are refused) it contracts the reference
   tensor with the geometry tensor on the tensor cores instead (tcgen05,
   half-precision limb pairs of the FP64 geometry, FP32 accumulation: about
   3e-7 of the entries' scale).  Its waits on the tensor core are bounded;
   *status = 1 reports that one ran out (the outputs of that call are NaN),
   0 that none has.  Synchronises the device.  No counterpart in the
   reference. */
int db2_tensor_core_status(int* status);
/* Vector-Jacobian product of (A(kappa), b(kappa)) for a = kappa grad.grad
   (P1 kappa) and L = f v dx, or the kappa-weighted load
   constant[0] * kappa f v dx when L->coeff is DB2_COEFF_P1_KAPPA (also
   DB2_COEFF_P1_SCALED, with constant[0] ignored, for earlier callers):
   dkappa[Nv] = sum gA*dA/dkappa + sum gb*db/dkappa.  gA[nnz], gb[N] device (gb may be NULL).  This is the
   assembly of UFL's derivative(a, kappa) form (the reference's
   python/test/unit/fem/test_coordinate_derivative.py style check). */
int db2_vjp_kappa(db2_pattern P, const db2_form* a, const double* kappa, const db2_form* L,
                  const double* f, const double* gA, const double* gb, int precision,
                  double* dkappa, void* stream);

/* Allocation-free variant of db2_vjp_kappa (no counterpart in the
   reference).  For callers that cannot let a library allocate device memory
   at call time -- applications whose device memory belongs to their own pool
   allocator, or loops with streams in flight that cudaMalloc's implicit
   synchronisation would stall.  Same arguments and result as
   db2_vjp_kappa, but the work array is a fixed array inside the library:
   at most 2^21 doubles, i.e. cells * (tdim + 1) <= 2097152 (524,288
   tetrahedra / 699,050 triangles); larger patterns fail with DB2_ERR_SHAPE.
   It calls no cudaMalloc/cudaFree and loads nothing: the pattern must
   already be resident on the current device (after any assembly with it, or
   db2_pattern_csr_device).  Making a pattern resident sets the array up on
   that device (cudaGetSymbolAddress, which with lazy module loading is when
   the 16 MiB reach the device) and loads the adjoint kernels; the device
   holds the array from then until the process exits.  All calls share the
   one array, so calls that overlap on the GPU (other streams, other
   threads) race; order them on one stream. */
int db2_vjp_kappa_noalloc(db2_pattern P, const db2_form* a, const double* kappa,
                          const db2_form* L, const double* f, const double* gA,
                          const double* gb, int precision, double* dkappa, void* stream);

/* ---- batched multi-mesh assembly -------------------------------------- */
/* A batch of patterns (any element/space mix) assembled by ONE persistent
   launch.  kappa pointers (device, one P1 field per member) and output
   pointers are fixed at creation so that the launch can be captured in a
   CUDA graph.  tile_nodes/seg_cap_bytes/ctas_per_sm = 0 choose defaults
   (the autotuner in dolfin_b200.batch chooses explicit values). */
int db2_batch_create(int count, const db2_pattern* patterns, const db2_form* forms,
                     const double* const* kappas, double* const* vals,
                     int tile_nodes, int seg_cap_bytes, int ctas_per_sm, db2_batch* out);
int db2_batch_info(db2_batch B, int64_t* tiles, int64_t* cells, int* ctas);
/* One persistent launch over every tile of every member (precision as above). */
int db2_batch_assemble(db2_batch B, int precision, void* stream);
/* Reference path: one launch per member, in member order. */
int db2_batch_assemble_loop(db2_batch B, int precision, void* stream);
int db2_batch_destroy(db2_batch B);

#ifdef __cplusplus
}
#endif
#endif /* DOLFIN_B200_H */
