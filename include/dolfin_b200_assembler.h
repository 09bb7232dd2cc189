/*
 * dolfin_b200_assembler.h -- C++ drop-in classes over the engine's C ABI.
 *
 * GpuAssembler and GpuSystemAssembler keep the call shapes of DOLFIN's
 *   void Assembler::assemble(GenericTensor& A, const Form& a)
 *       (dolfin/fem/Assembler.h:66, flags of AssemblerBase.h:46-67), and
 *   SystemAssembler(std::shared_ptr<const Form> a, std::shared_ptr<const Form> L,
 *                   std::vector<std::shared_ptr<const DirichletBC>> bcs)
 *   void SystemAssembler::assemble(GenericMatrix& A, GenericVector& b)
 *       (dolfin/fem/SystemAssembler.h:63-84),
 * on small stand-ins for the DOLFIN objects they take (Mesh, FunctionSpace,
 * Function, Form, GenericTensor/Matrix/Vector, DirichletBC).  Everything
 * below goes through include/dolfin_b200.h only; the implementation is
 * dolfin_b200/csrc/shim/assembler.cpp, built as libdolfin_b200_cpp.so
 * (link with -ldolfin_b200_cpp -ldolfin_b200 -lcudart).
 *
 * Forms: FFC generates DOLFIN's forms; here the named forms the engine
 * provides are built by the functions of namespace forms (the UFL of each is
 * given beside it).  Tensors hold their values in device memory; data() /
 * get_local() copy them to the host like EigenMatrix::data() and
 * GenericVector::get_local().  Failures throw std::runtime_error with the
 * "*** Error: Unable to <task>.\n*** Reason:  <reason>" text of
 * dolfin_error() (dolfin/log/log.cpp:129).
 */
#ifndef DOLFIN_B200_ASSEMBLER_H
#define DOLFIN_B200_ASSEMBLER_H

#include <cstddef>
#include <cstdint>
#include <functional>
#include <memory>
#include <string>
#include <tuple>
#include <vector>

#include "dolfin_b200.h"

namespace dolfin_b200 {

// dolfin_error(file, task, reason) as an exception.
[[noreturn]] void dolfin_error(const std::string& file, const std::string& task,
                               const std::string& reason);

// dolfin::Mesh (triangles or tetrahedra, cell vertex lists sorted).
class Mesh {
 public:
  Mesh(int tdim, const std::vector<double>& coordinates, const std::vector<uint32_t>& cells);
  static std::shared_ptr<Mesh> UnitCube(int nx, int ny, int nz);   // BoxMesh::build_tet
  static std::shared_ptr<Mesh> UnitSquare(int nx, int ny, const std::string& diagonal = "right");
  ~Mesh();
  Mesh(const Mesh&) = delete;
  Mesh& operator=(const Mesh&) = delete;
  int topology_dim() const { return tdim_; }
  std::size_t num_vertices() const { return std::size_t(nv_); }
  std::size_t num_cells() const { return std::size_t(nc_); }
  std::vector<double> coordinates() const;
  std::vector<uint32_t> cells() const;
  void set_coordinates(const std::vector<double>& x);
  db2_mesh handle() const { return h_; }

 private:
  explicit Mesh(db2_mesh h);
  db2_mesh h_ = nullptr;
  int tdim_ = 0;
  int64_t nv_ = 0, nc_ = 0;
};

// dolfin::FunctionSpace of continuous Lagrange elements (scalar or vector),
// natural dof numbering; owns its sparsity pattern(s).
class FunctionSpace {
 public:
  FunctionSpace(std::shared_ptr<const Mesh> mesh, int degree, int value_size = 1);
  ~FunctionSpace();
  FunctionSpace(const FunctionSpace&) = delete;
  FunctionSpace& operator=(const FunctionSpace&) = delete;
  std::shared_ptr<const Mesh> mesh() const { return mesh_; }
  int degree() const { return degree_; }
  int value_size() const { return vsize_; }
  std::size_t dim() const { return std::size_t(dim_); }
  int ndofs_per_cell() const { return k_; }
  std::vector<int32_t> cell_dofs_all() const;      // DofMap::cell_dofs of every cell
  db2_space handle() const { return h_; }
  db2_pattern pattern(bool keep_diagonal = false) const;  // built on first use

 private:
  std::shared_ptr<const Mesh> mesh_;
  db2_space h_ = nullptr;
  int degree_, vsize_, k_ = 0;
  int64_t dim_ = 0;
  mutable db2_pattern pattern_[2] = {nullptr, nullptr};
};

// A P1 coefficient (dolfin::Function on a scalar P1 space): vertex values
// held in device memory.
class Function {
 public:
  Function(std::shared_ptr<const FunctionSpace> V, const std::vector<double>& values);
  ~Function();
  Function(const Function&) = delete;
  Function& operator=(const Function&) = delete;
  std::shared_ptr<const FunctionSpace> function_space() const { return V_; }
  void set_values(const std::vector<double>& values);
  const double* device_values() const { return d_; }

 private:
  std::shared_ptr<const FunctionSpace> V_;
  double* d_ = nullptr;
};

// A named form on a space (the role of an FFC-generated dolfin::Form): one
// cell (dx) part and/or one exterior-facet (ds) part, each a kernel of the
// engine with its coefficient.
class Form {
 public:
  struct Part {
    db2_form desc;
    std::shared_ptr<const Function> w;   // P1 coefficient, or nullptr
    const double* values() const;        // device values of w, or nullptr
  };
  Form(int rank, std::shared_ptr<const FunctionSpace> V, std::vector<Part> parts);
  int rank() const { return rank_; }
  std::shared_ptr<const FunctionSpace> function_space() const { return V_; }
  const Part* cell_part() const;    // the dx part, or nullptr
  const Part* facet_part() const;   // the ds part, or nullptr

 private:
  int rank_;
  std::shared_ptr<const FunctionSpace> V_;
  std::vector<Part> parts_;
};

namespace forms {
// kappa*inner(grad(u), grad(v))*dx, kappa a Constant or a P1 Function
std::shared_ptr<Form> Diffusion(std::shared_ptr<const FunctionSpace> V, double kappa = 1.0);
std::shared_ptr<Form> Diffusion(std::shared_ptr<const FunctionSpace> V,
                                std::shared_ptr<const Function> kappa);
// f*v*dx (scalar V) or inner(f, v)*dx (vector V, f a constant vector)
std::shared_ptr<Form> Load(std::shared_ptr<const FunctionSpace> V, std::vector<double> f);
std::shared_ptr<Form> Load(std::shared_ptr<const FunctionSpace> V, std::shared_ptr<const Function> f);
// inner(2 mu eps(u) + lmbda tr(eps(u)) I, eps(v))*dx on a 3D vector space
std::shared_ptr<Form> Elasticity(std::shared_ptr<const FunctionSpace> V, double mu, double lmbda);
// w*u*v*ds and g*v*ds (scalar V; w, g Constants)
std::shared_ptr<Form> BoundaryMass(std::shared_ptr<const FunctionSpace> V, double w);
std::shared_ptr<Form> BoundaryLoad(std::shared_ptr<const FunctionSpace> V, double g);
// a + b: a dx form plus a ds form of the same rank on the same space
std::shared_ptr<Form> Sum(std::shared_ptr<const Form> a, std::shared_ptr<const Form> b);
}  // namespace forms

// dolfin::GenericTensor: the part of its interface assembly uses
// (dolfin/la/GenericTensor.h:58-110).
class GenericTensor {
 public:
  virtual ~GenericTensor() = default;
  virtual bool empty() const = 0;
  virtual void zero() = 0;
  virtual void apply(const std::string& mode) = 0;
  virtual std::size_t size(std::size_t dim) const = 0;
  virtual std::size_t rank() const = 0;
};

// CSR matrix in device memory on a pattern of the engine (EigenMatrix's
// RowMajor SparseMatrix<double, int> layout).
class Matrix : public GenericTensor {
 public:
  Matrix() = default;
  ~Matrix() override;
  Matrix(const Matrix&) = delete;
  Matrix& operator=(const Matrix&) = delete;
  void init(db2_pattern P);
  bool empty() const override { return P_ == nullptr; }
  void zero() override;
  void apply(const std::string&) override {}
  std::size_t size(std::size_t dim) const override;
  std::size_t rank() const override { return 2; }
  std::size_t nnz() const { return std::size_t(nnz_); }
  db2_pattern pattern() const { return P_; }
  double* device_values() { return vals_; }
  // host copies (row pointers, columns, values, nnz) as EigenMatrix::data()
  std::tuple<std::vector<int32_t>, std::vector<int32_t>, std::vector<double>> data() const;

 private:
  db2_pattern P_ = nullptr;
  int64_t nrows_ = 0, nnz_ = 0;
  double* vals_ = nullptr;
};

class Vector : public GenericTensor {
 public:
  explicit Vector(std::size_t n = 0);
  ~Vector() override;
  Vector(const Vector&) = delete;
  Vector& operator=(const Vector&) = delete;
  void init(std::size_t n);
  bool empty() const override { return n_ == 0; }
  void zero() override;
  void apply(const std::string&) override {}
  std::size_t size(std::size_t dim = 0) const override { return dim == 0 ? n_ : 1; }
  std::size_t rank() const override { return 1; }
  double* device_values() { return x_; }
  void get_local(std::vector<double>& values) const;

 private:
  std::size_t n_ = 0;
  double* x_ = nullptr;
};

// dolfin::DirichletBC with the topological method: the dofs of the closure
// of the exterior facets the marker accepts (all of them for
// "on_boundary"; a callable sees each facet vertex and the facet midpoint).
class DirichletBC {
 public:
  using Marker = std::function<bool(const double* x, bool on_boundary)>;
  DirichletBC(std::shared_ptr<const FunctionSpace> V, double value,
              const std::string& where = "on_boundary");
  DirichletBC(std::shared_ptr<const FunctionSpace> V, double value, Marker marker);
  std::shared_ptr<const FunctionSpace> function_space() const { return V_; }
  const std::vector<int64_t>& dofs() const { return dofs_; }
  double value() const { return value_; }

 private:
  void build(const Marker& marker);
  std::shared_ptr<const FunctionSpace> V_;
  double value_;
  std::vector<int64_t> dofs_;
};

// dolfin::Assembler (dolfin/fem/Assembler.h) on the GPU.
class GpuAssembler {
 public:
  bool add_values = false;       // AssemblerBase::add_values
  bool finalize_tensor = true;   // AssemblerBase::finalize_tensor (values are final anyway)
  bool keep_diagonal = false;    // AssemblerBase::keep_diagonal
  int precision = DB2_FP64;      // DB2_FP32_CONTRACT: FP32 reference-tensor contraction
  void* stream = nullptr;        // cudaStream_t; nullptr = the legacy default stream

  // Assembler::assemble(GenericTensor& A, const Form& a): a Matrix for a
  // bilinear form, a Vector for a linear form (dx and ds forms).
  void assemble(GenericTensor& A, const Form& a);
  // double assemble(const Form&) is not provided for the named forms.
};

// dolfin::SystemAssembler (dolfin/fem/SystemAssembler.h) on the GPU: A and b
// in one pass, Dirichlet conditions applied symmetrically per cell.
class GpuSystemAssembler {
 public:
  GpuSystemAssembler(std::shared_ptr<const Form> a, std::shared_ptr<const Form> L,
                     std::vector<std::shared_ptr<const DirichletBC>> bcs = {});
  bool keep_diagonal = false;
  int precision = DB2_FP64;
  void* stream = nullptr;
  void assemble(Matrix& A, Vector& b);
  void assemble(Matrix& A);
  void assemble(Vector& b);

 private:
  std::shared_ptr<const Form> a_, L_;
  std::vector<std::shared_ptr<const DirichletBC>> bcs_;
};

}  // namespace dolfin_b200

#endif  // DOLFIN_B200_ASSEMBLER_H
