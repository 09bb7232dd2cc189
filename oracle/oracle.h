/*
 * oracle.h -- C interface of the CPU oracle.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is a plain CPU restatement of
 * DOLFIN 2019.1's finite-element assembly path (mesh generation and
 * ordering, entity numbering, natural UFC dofmaps, sparsity pattern,
 * Assembler::assemble_cells, SystemAssembler::cell_wise_assembly) used as
 * the correctness checker of the CUDA engine.  Only tests/, the smoke check
 * and the CPU-baseline leg of bench.py may load it.  The product library
 * (dolfin_b200) never links or calls it.
 *
 * Parity anchor: the reference itself cannot be built here (it needs FFC,
 * UFL, Boost, Eigen and MPI).  The restatement is pinned against the
 * known-answer tests shipped in the reference's own test-suite
 * (python/test/unit/fem/test_assembler.py, test_system_assembler.py,
 * python/test/unit/la/test_matrix.py); see tests/test_oracle_golden.py.
 */
#ifndef DOLFIN_B200_ORACLE_H
#define DOLFIN_B200_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- forms ------------------------------------------------------------ */
enum orc_form_kind {
  ORC_DIFFUSION = 1,   /* a = kappa * inner(grad(u), grad(v)) * dx            */
  ORC_MASS = 2,        /* a = u * v * dx                                      */
  ORC_LOAD = 3,        /* L = f * v * dx  (scalar f, or constant vector f)    */
  ORC_ELASTICITY = 4,  /* a = inner(sigma(u), epsilon(v)) * dx,
                          sigma = 2 mu eps + lmbda tr(eps) I                  */
  ORC_DIV_P = 5,       /* a = div(v) * p * dx     (v vector test, p trial)    */
  ORC_GRADP_V = 6,     /* a = inner(grad(p), v) * dx                          */
  ORC_FUNCTIONAL = 7,  /* M = coeff * dx, coeff = const, P1 field or x[i]     */
  /* exterior facet integrals (Assembler::assemble_exterior_facets)           */
  ORC_FACET_MASS = 8,       /* a = coeff * u * v * ds   (scalar spaces)       */
  ORC_FACET_LOAD = 9,       /* L = coeff * v * ds, or inner(c, v) * ds        */
  ORC_FACET_FUNCTIONAL = 10 /* M = coeff * ds                                 */
};

enum orc_coeff_kind {
  ORC_COEFF_NONE = 0,   /* coefficient == 1                                   */
  ORC_COEFF_CONST = 1,  /* Constant: value(s) in c[]                          */
  ORC_COEFF_P1 = 2,     /* P1 Function given by its vertex values             */
  ORC_COEFF_X0 = 3,     /* SpatialCoordinate x[i], i = (int)c[1] (0 default)  */
  ORC_COEFF_P1_TIMES_P1 = 4 /* product of two P1 fields (w, w2)               */
};

enum orc_family { ORC_CG = 0, ORC_DG = 1 };

typedef struct {
  int kind;                 /* orc_form_kind                                  */
  int tdim, gdim;           /* cell: 1 interval, 2 triangle, 3 tetrahedron    */
  int family0, degree0, vsize0;  /* test space  (rank >= 1)                   */
  int family1, degree1, vsize1;  /* trial space (rank 2)                      */
  int coeff;                /* orc_coeff_kind                                 */
  double c[3];              /* constant values                                */
  double mu, lmbda;         /* elasticity constants                           */
} orc_form;

/* ---- meshes (dolfin/generation) --------------------------------------- */
/* UnitCubeMesh(nx,ny,nz) == BoxMesh((0,0,0),(1,1,1)): coords[(nx+1)(ny+1)(nz+1)*3],
   cells[6*nx*ny*nz*4] (vertices sorted ascending, as after MeshEditor::close) */
int orc_box_mesh(int nx, int ny, int nz, double* coords, uint32_t* cells);
/* UnitSquareMesh(nx,ny,diagonal): diagonal 0 = "right", 1 = "left",
   2 = "right/left", 3 = "left/right".  coords[(nx+1)(ny+1)*2], cells[2*nx*ny*3] */
int orc_rectangle_mesh(int nx, int ny, int diagonal, double* coords, uint32_t* cells);
/* UnitIntervalMesh(n): coords[n+1], cells[2n] */
int orc_interval_mesh(int n, double* coords, uint32_t* cells);

/* ---- topology (TopologyComputation::compute_entities_by_key_matching) -- */
/* Number of edges; fills cell_edges[nc * nedge_per_cell] (local edge order
   of TetrahedronCell/TriangleCell::create_entities) and, if non-NULL,
   edge_vertices[ne*2]. */
int64_t orc_edges(int tdim, int64_t nc, const uint32_t* cells,
                  uint32_t* cell_edges, uint32_t* edge_vertices);

/* Exterior facets (facets with one incident cell), in facet-number order
   (key order, as compute_entities_by_key_matching numbers them): the cell of
   each and its local facet index (facet i is opposite local vertex i).
   Arrays hold up to nc*(tdim+1) entries; returns the count. */
int64_t orc_exterior_facets(int tdim, int64_t nc, const uint32_t* cells,
                            uint32_t* facet_cell, int32_t* facet_local);

/* ---- dofmap (DofMapBuilder::build with reorder_dofs_serial = false) --- */
/* Returns the global dimension; fills cell_dofs[nc * ndofs_per_cell]. */
int64_t orc_dofmap(int family, int degree, int vsize, int tdim,
                   int64_t nv, int64_t nc, const uint32_t* cells,
                   int32_t* cell_dofs);
int orc_ndofs_per_cell(int family, int degree, int vsize, int tdim);
/* DofMapBuilder::build with reorder_dofs_serial = true and
   dof_ordering_library = "Boost" (CG only): node graph with dolfin::Set
   insertion, Boost's reverse Cuthill-McKee, dofs bs*node + c.  node_new may
   be NULL. */
int64_t orc_dofmap_reordered(int degree, int vsize, int tdim, int64_t nv, int64_t nc,
                             const uint32_t* cells, int32_t* cell_dofs, int32_t* node_new);

/* ---- sparsity (SparsityPatternBuilder::build + EigenMatrix::init) ----- */
typedef struct orc_csr orc_csr;
orc_csr* orc_sparsity(int64_t nrows, int64_t ncols, int64_t nc,
                      int k0, const int32_t* dofs0, int k1, const int32_t* dofs1,
                      int keep_diagonal);
int64_t orc_csr_nnz(const orc_csr* p);
void orc_csr_copy(const orc_csr* p, int32_t* rowptr, int32_t* cols);
void orc_csr_free(orc_csr* p);

/* ---- assembly (Assembler::assemble_cells, EigenMatrix/EigenVector::add) */
/* Element tensor of one cell: coordinate_dofs vertex-major (as
   Cell::get_coordinate_dofs), w = coefficient vertex values of the cell. */
int orc_element_tensor(const orc_form* f, const double* coordinate_dofs,
                       const double* w, const double* w2, double* A);

/* Matrix assembly into a preallocated sorted CSR (rowptr/cols); vals is
   zeroed first unless add_values.  w/w2 are P1 vertex fields (or NULL).
   cells selects a subset when first_cell/ncells_used restrict it. */
int orc_assemble_matrix(const orc_form* f, int64_t nv, const double* coords,
                        int64_t nc, const uint32_t* cells,
                        const int32_t* dofs0, const int32_t* dofs1,
                        const double* w, const double* w2,
                        int64_t nrows, const int32_t* rowptr, const int32_t* cols,
                        double* vals, int add_values);
int orc_assemble_vector(const orc_form* f, int64_t nv, const double* coords,
                        int64_t nc, const uint32_t* cells, const int32_t* dofs0,
                        const double* w, const double* w2,
                        int64_t n, double* b, int add_values);
double orc_assemble_scalar(const orc_form* f, int64_t nv, const double* coords,
                           int64_t nc, const uint32_t* cells, const double* w);

/* SystemAssembler(a, L, bc).assemble(A, b): cell-wise assembly with the
   symmetric Dirichlet modification SystemAssembler::apply_bc.  bc_dofs
   (sorted, unique) carry bc_vals. */
int orc_assemble_system(const orc_form* a, const orc_form* L, int64_t nv,
                        const double* coords, int64_t nc, const uint32_t* cells,
                        const int32_t* dofs, const double* wa, const double* wL,
                        int64_t nbc, const int32_t* bc_dofs, const double* bc_vals,
                        int64_t n, const int32_t* rowptr, const int32_t* cols,
                        double* vals, double* b);

/* Same with exterior facet integrals a_ds / L_ds (either may be NULL) added
   to each cell tensor before apply_bc, as SystemAssembler::cell_wise_assembly
   does for the exterior facets of the cell (SystemAssembler.cpp:417-470). */
int orc_assemble_system_ds(const orc_form* a, const orc_form* a_ds, const orc_form* L,
                           const orc_form* L_ds, int64_t nv, const double* coords,
                           int64_t nc, const uint32_t* cells, const int32_t* dofs,
                           const double* wa, const double* wa_ds, const double* wL,
                           const double* wL_ds, int64_t nbc, const int32_t* bc_dofs,
                           const double* bc_vals, int64_t n, const int32_t* rowptr,
                           const int32_t* cols, double* vals, double* b);

/* Vertices on the boundary of a UnitCube/UnitSquare box mesh (the dofs of
   DirichletBC(V, g, "on_boundary") for P1); returns count. */
int64_t orc_boundary_vertices(int gdim, int64_t nv, const double* coords,
                              int32_t* out);

/* Adjoint reference: the derivative form of a = kappa*grad(u).grad(v)*dx
   (and of L = kappa*f*v*dx when load_has_kappa) with respect to the P1
   field kappa, contracted with upstream gradients gA (CSR shaped) and gb:
   dkappa[v] = sum_ij gA_ij * d a_ij / d kappa_v + sum_i gb_i * d L_i / d kappa_v. */
int orc_vjp_diffusion(const orc_form* a, int64_t nv, const double* coords,
                      int64_t nc, const uint32_t* cells, const int32_t* dofs,
                      const int32_t* rowptr, const int32_t* cols, const double* gA,
                      const double* f, const double* gb, int load_has_kappa,
                      double* dkappa);

/* Quadrature self-check: integral of x^a y^b z^c over the reference simplex. */
double orc_quadrature_monomial(int tdim, int degree, int a, int b, int c);

#ifdef __cplusplus
}
#endif
#endif
