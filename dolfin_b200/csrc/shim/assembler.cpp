// assembler.cpp -- the C++ drop-in classes (include/dolfin_b200_assembler.h).
//
// Host-side glue only: every engine operation goes through the C ABI of
// include/dolfin_b200.h, the way a binding in DOLFIN's own tree would call
// it; device buffers of tensors and coefficients are plain cudaMalloc
// allocations owned by these objects.
#include "../../../include/dolfin_b200_assembler.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <set>
#include <stdexcept>

namespace dolfin_b200 {

void dolfin_error(const std::string& file, const std::string& task, const std::string& reason) {
  throw std::runtime_error("\n*** Error:   Unable to " + task + ".\n*** Reason:  " + reason +
                           "\n*** Where:   This error was encountered inside " + file + ".");
}

namespace {

void check(int rc, const char* task) {
  if (rc != DB2_OK) dolfin_error("assembler.cpp", task, db2_last_error());
}

void check_cuda(cudaError_t e, const char* task) {
  if (e != cudaSuccess) dolfin_error("assembler.cpp", task, cudaGetErrorString(e));
}

template <typename T>
T* device_alloc(std::size_t n, const char* task) {
  void* p = nullptr;
  if (n) check_cuda(cudaMalloc(&p, n * sizeof(T)), task);
  return static_cast<T*>(p);
}

db2_form make_desc(int kind, int coeff, const double* c = nullptr, int nc = 0, double mu = 0.0,
                   double lmbda = 0.0) {
  db2_form f;
  std::memset(&f, 0, sizeof(f));
  f.kind = kind;
  f.coeff = coeff;
  for (int i = 0; i < nc && i < 3; ++i) f.constant[i] = c[i];
  f.mu = mu;
  f.lmbda = lmbda;
  return f;
}

bool facet_kind(int kind) { return kind == DB2_FORM_FACET_MASS || kind == DB2_FORM_FACET_LOAD; }

// UFC local edges (TetrahedronCell.cpp:119-124, TriangleCell.cpp:106-108)
const int kTetE[6][2] = {{2, 3}, {1, 3}, {1, 2}, {0, 3}, {0, 2}, {0, 1}};
const int kTriE[3][2] = {{1, 2}, {0, 2}, {0, 1}};

}  // namespace

// ---- Mesh -------------------------------------------------------------------
Mesh::Mesh(db2_mesh h) : h_(h) {
  check(db2_mesh_info(h_, &tdim_, &nv_, &nc_), "read mesh size");
}

Mesh::Mesh(int tdim, const std::vector<double>& x, const std::vector<uint32_t>& cells) {
  const int64_t nv = int64_t(x.size()) / std::max(tdim, 1);
  const int64_t nc = int64_t(cells.size()) / (tdim + 1);
  check(db2_mesh_create(tdim, nv, x.data(), nc, cells.data(), &h_), "create mesh");
  check(db2_mesh_info(h_, &tdim_, &nv_, &nc_), "read mesh size");
}

std::shared_ptr<Mesh> Mesh::UnitCube(int nx, int ny, int nz) {
  db2_mesh h = nullptr;
  check(db2_mesh_unit_cube(nx, ny, nz, &h), "create UnitCubeMesh");
  return std::shared_ptr<Mesh>(new Mesh(h));
}

std::shared_ptr<Mesh> Mesh::UnitSquare(int nx, int ny, const std::string& diagonal) {
  const int d = diagonal == "right" ? 0 : diagonal == "left" ? 1 : diagonal == "right/left" ? 2
              : diagonal == "left/right" ? 3 : -1;
  if (d < 0) dolfin_error("assembler.cpp", "create UnitSquareMesh", "unknown diagonal " + diagonal);
  db2_mesh h = nullptr;
  check(db2_mesh_unit_square(nx, ny, d, &h), "create UnitSquareMesh");
  return std::shared_ptr<Mesh>(new Mesh(h));
}

Mesh::~Mesh() {
  if (h_) db2_mesh_destroy(h_);
}

std::vector<double> Mesh::coordinates() const {
  std::vector<double> x(std::size_t(nv_) * tdim_);
  check(db2_mesh_copy(h_, x.data(), nullptr), "copy coordinates");
  return x;
}

std::vector<uint32_t> Mesh::cells() const {
  std::vector<uint32_t> c(std::size_t(nc_) * (tdim_ + 1));
  check(db2_mesh_copy(h_, nullptr, c.data()), "copy cells");
  return c;
}

void Mesh::set_coordinates(const std::vector<double>& x) {
  if (x.size() != std::size_t(nv_) * tdim_)
    dolfin_error("assembler.cpp", "set coordinates", "wrong number of values");
  check(db2_mesh_set_coordinates(h_, x.data()), "set coordinates");
}

// ---- FunctionSpace ----------------------------------------------------------
FunctionSpace::FunctionSpace(std::shared_ptr<const Mesh> mesh, int degree, int value_size)
    : mesh_(std::move(mesh)), degree_(degree), vsize_(value_size) {
  check(db2_space_create(mesh_->handle(), degree, value_size, &h_), "create function space");
  check(db2_space_info(h_, &k_, &dim_), "read function space size");
}

FunctionSpace::~FunctionSpace() {
  for (auto& p : pattern_)
    if (p) db2_pattern_destroy(p);
  if (h_) db2_space_destroy(h_);
}

std::vector<int32_t> FunctionSpace::cell_dofs_all() const {
  std::vector<int32_t> d(mesh_->num_cells() * std::size_t(k_));
  check(db2_space_cell_dofs(h_, d.data()), "copy cell dofs");
  return d;
}

db2_pattern FunctionSpace::pattern(bool keep_diagonal) const {
  db2_pattern& p = pattern_[keep_diagonal ? 1 : 0];
  if (!p) check(db2_pattern_create(h_, keep_diagonal ? 1 : 0, &p), "build sparsity pattern");
  return p;
}

// ---- Function ---------------------------------------------------------------
Function::Function(std::shared_ptr<const FunctionSpace> V, const std::vector<double>& values)
    : V_(std::move(V)) {
  if (V_->degree() != 1 || V_->value_size() != 1)
    dolfin_error("assembler.cpp", "create coefficient", "coefficients are scalar P1 Functions");
  d_ = device_alloc<double>(V_->dim(), "allocate coefficient");
  set_values(values);
}

Function::~Function() {
  if (d_) cudaFree(d_);
}

void Function::set_values(const std::vector<double>& values) {
  if (values.size() != V_->dim())
    dolfin_error("assembler.cpp", "set coefficient values", "wrong number of values");
  check_cuda(cudaMemcpy(d_, values.data(), values.size() * sizeof(double), cudaMemcpyHostToDevice),
             "upload coefficient");
}

// ---- Form -------------------------------------------------------------------
const double* Form::Part::values() const { return w ? w->device_values() : nullptr; }

Form::Form(int rank, std::shared_ptr<const FunctionSpace> V, std::vector<Part> parts)
    : rank_(rank), V_(std::move(V)), parts_(std::move(parts)) {
  int ncell = 0, nfacet = 0;
  for (const Part& p : parts_) (facet_kind(p.desc.kind) ? nfacet : ncell)++;
  if (ncell > 1 || nfacet > 1 || parts_.empty())
    dolfin_error("assembler.cpp", "create form", "a form has one dx part and/or one ds part");
  for (const Part& p : parts_)
    if (p.w && p.w->function_space()->mesh() != V_->mesh())
      dolfin_error("assembler.cpp", "create form", "coefficient and form live on different meshes");
}

const Form::Part* Form::cell_part() const {
  for (const Part& p : parts_)
    if (!facet_kind(p.desc.kind)) return &p;
  return nullptr;
}

const Form::Part* Form::facet_part() const {
  for (const Part& p : parts_)
    if (facet_kind(p.desc.kind)) return &p;
  return nullptr;
}

namespace forms {
using SpacePtr = std::shared_ptr<const FunctionSpace>;
using FunctionPtr = std::shared_ptr<const Function>;

std::shared_ptr<Form> Diffusion(SpacePtr V, double kappa) {
  const int coeff = kappa == 1.0 ? DB2_COEFF_NONE : DB2_COEFF_CONSTANT;
  return std::make_shared<Form>(2, V, std::vector<Form::Part>{
      {make_desc(DB2_FORM_DIFFUSION, coeff, &kappa, 1), nullptr}});
}

std::shared_ptr<Form> Diffusion(SpacePtr V, FunctionPtr kappa) {
  return std::make_shared<Form>(2, V, std::vector<Form::Part>{
      {make_desc(DB2_FORM_DIFFUSION, DB2_COEFF_P1), kappa}});
}

std::shared_ptr<Form> Load(SpacePtr V, std::vector<double> f) {
  if (f.size() != std::size_t(V->value_size()))
    dolfin_error("assembler.cpp", "create load form", "the load has the wrong number of components");
  return std::make_shared<Form>(1, V, std::vector<Form::Part>{
      {make_desc(DB2_FORM_LOAD, DB2_COEFF_CONSTANT, f.data(), int(f.size())), nullptr}});
}

std::shared_ptr<Form> Load(SpacePtr V, FunctionPtr f) {
  return std::make_shared<Form>(1, V, std::vector<Form::Part>{
      {make_desc(DB2_FORM_LOAD, DB2_COEFF_P1), f}});
}

std::shared_ptr<Form> Elasticity(SpacePtr V, double mu, double lmbda) {
  return std::make_shared<Form>(2, V, std::vector<Form::Part>{
      {make_desc(DB2_FORM_ELASTICITY, DB2_COEFF_NONE, nullptr, 0, mu, lmbda), nullptr}});
}

std::shared_ptr<Form> BoundaryMass(SpacePtr V, double w) {
  return std::make_shared<Form>(2, V, std::vector<Form::Part>{
      {make_desc(DB2_FORM_FACET_MASS, w == 1.0 ? DB2_COEFF_NONE : DB2_COEFF_CONSTANT, &w, 1), nullptr}});
}

std::shared_ptr<Form> BoundaryLoad(SpacePtr V, double g) {
  return std::make_shared<Form>(1, V, std::vector<Form::Part>{
      {make_desc(DB2_FORM_FACET_LOAD, g == 1.0 ? DB2_COEFF_NONE : DB2_COEFF_CONSTANT, &g, 1), nullptr}});
}

std::shared_ptr<Form> Sum(std::shared_ptr<const Form> a, std::shared_ptr<const Form> b) {
  if (a->rank() != b->rank() || a->function_space() != b->function_space())
    dolfin_error("assembler.cpp", "add forms", "the forms differ in rank or space");
  std::vector<Form::Part> parts;
  for (const Form* f : {a.get(), b.get()}) {
    if (f->cell_part()) parts.push_back(*f->cell_part());
    if (f->facet_part()) parts.push_back(*f->facet_part());
  }
  return std::make_shared<Form>(a->rank(), a->function_space(), parts);
}
}  // namespace forms

// ---- tensors ----------------------------------------------------------------
Matrix::~Matrix() {
  if (vals_) cudaFree(vals_);
}

void Matrix::init(db2_pattern P) {
  if (vals_) cudaFree(vals_);
  vals_ = nullptr;
  P_ = P;
  check(db2_pattern_info(P_, &nrows_, &nnz_), "read sparsity pattern");
  vals_ = device_alloc<double>(std::size_t(nnz_), "allocate matrix values");
  zero();
}

void Matrix::zero() {
  if (nnz_) check_cuda(cudaMemset(vals_, 0, std::size_t(nnz_) * sizeof(double)), "zero matrix");
}

std::size_t Matrix::size(std::size_t) const { return std::size_t(nrows_); }

std::tuple<std::vector<int32_t>, std::vector<int32_t>, std::vector<double>> Matrix::data() const {
  std::vector<int32_t> rp(static_cast<std::size_t>(nrows_) + 1), cols(static_cast<std::size_t>(nnz_));
  std::vector<double> v(static_cast<std::size_t>(nnz_));
  check(db2_pattern_csr_host(P_, rp.data(), cols.data()), "copy sparsity pattern");
  check_cuda(cudaMemcpy(v.data(), vals_, v.size() * sizeof(double), cudaMemcpyDeviceToHost),
             "copy matrix values");
  return {std::move(rp), std::move(cols), std::move(v)};
}

Vector::Vector(std::size_t n) { init(n); }

Vector::~Vector() {
  if (x_) cudaFree(x_);
}

void Vector::init(std::size_t n) {
  if (x_) cudaFree(x_);
  x_ = nullptr;
  n_ = n;
  x_ = device_alloc<double>(n, "allocate vector");
  zero();
}

void Vector::zero() {
  if (n_) check_cuda(cudaMemset(x_, 0, n_ * sizeof(double)), "zero vector");
}

void Vector::get_local(std::vector<double>& values) const {
  values.resize(n_);
  check_cuda(cudaMemcpy(values.data(), x_, n_ * sizeof(double), cudaMemcpyDeviceToHost),
             "copy vector values");
}

// ---- DirichletBC --------------------------------------------------------------
DirichletBC::DirichletBC(std::shared_ptr<const FunctionSpace> V, double value, const std::string& where)
    : V_(std::move(V)), value_(value) {
  if (where != "on_boundary")
    dolfin_error("assembler.cpp", "create boundary condition", "markers: \"on_boundary\" or a callable");
  build(nullptr);
}

DirichletBC::DirichletBC(std::shared_ptr<const FunctionSpace> V, double value, Marker marker)
    : V_(std::move(V)), value_(value) {
  build(marker);
}

void DirichletBC::build(const Marker& marker) {
  const Mesh& m = *V_->mesh();
  const int D = m.topology_dim(), nvc = D + 1;
  int64_t nf = 0;
  check(db2_mesh_num_exterior_facets(m.handle(), &nf), "count exterior facets");
  std::vector<uint32_t> fcell(static_cast<std::size_t>(nf));
  std::vector<int32_t> flocal(static_cast<std::size_t>(nf));
  check(db2_mesh_exterior_facets(m.handle(), fcell.data(), flocal.data()), "copy exterior facets");
  const std::vector<uint32_t> cells = m.cells();
  const std::vector<double> x = marker ? m.coordinates() : std::vector<double>();
  const std::vector<int32_t> cd = V_->cell_dofs_all();
  const int vs = V_->value_size(), k = V_->ndofs_per_cell() / vs;
  const int64_t nn = int64_t(V_->dim()) / vs;
  const int(*E)[2] = D == 3 ? kTetE : kTriE;
  std::set<int64_t> nodes;
  for (int64_t i = 0; i < nf; ++i) {
    const uint32_t c = fcell[i];
    const int a = flocal[i];
    if (marker) {
      // every facet vertex and the facet midpoint must be accepted
      double mid[3] = {0, 0, 0};
      bool ok = true;
      for (int b = 0; b < nvc && ok; ++b) {
        if (b == a) continue;
        const double* p = &x[std::size_t(cells[std::size_t(c) * nvc + b]) * D];
        for (int r = 0; r < D; ++r) mid[r] += p[r] / D;
        ok = marker(p, true);
      }
      if (!ok || !marker(mid, true)) continue;
    }
    for (int b = 0; b < nvc; ++b)
      if (b != a) nodes.insert(cd[std::size_t(c) * vs * k + b]);  // component-0 dofs are nodes
    if (V_->degree() == 2)
      for (int e = 0; e < (D == 3 ? 6 : 3); ++e)
        if (E[e][0] != a && E[e][1] != a) nodes.insert(cd[std::size_t(c) * vs * k + nvc + e]);
  }
  for (int c = 0; c < vs; ++c)
    for (int64_t node : nodes) dofs_.push_back(c * nn + node);
}

// ---- assemblers ---------------------------------------------------------------
namespace {

void check_dims(const GenericTensor& T, const FunctionSpace& V) {
  // AssemblerBase::init_global_tensor (dolfin/fem/AssemblerBase.cpp:182-191)
  if (T.size(0) != V.dim())
    dolfin_error("AssemblerBase.cpp", "assemble form", "Dim 0 of tensor does not match form");
}

// Dirichlet dofs and values as device arrays (flags uint8, values f64).
struct BCArrays {
  uint8_t* flags = nullptr;
  double* vals = nullptr;
  ~BCArrays() {
    if (flags) cudaFree(flags);
    if (vals) cudaFree(vals);
  }
};

void bc_arrays(const std::vector<std::shared_ptr<const DirichletBC>>& bcs, std::size_t n, BCArrays& out) {
  std::vector<uint8_t> f(n, 0);
  std::vector<double> v(n, 0.0);
  for (const auto& bc : bcs)
    for (int64_t d : bc->dofs()) {
      f[std::size_t(d)] = 1;
      v[std::size_t(d)] = bc->value();
    }
  out.flags = device_alloc<uint8_t>(n, "allocate boundary flags");
  out.vals = device_alloc<double>(n, "allocate boundary values");
  check_cuda(cudaMemcpy(out.flags, f.data(), n, cudaMemcpyHostToDevice), "upload boundary flags");
  check_cuda(cudaMemcpy(out.vals, v.data(), n * sizeof(double), cudaMemcpyHostToDevice),
             "upload boundary values");
}

}  // namespace

void GpuAssembler::assemble(GenericTensor& A, const Form& a) {
  const FunctionSpace& V = *a.function_space();
  const Form::Part* parts[2] = {a.cell_part(), a.facet_part()};
  if (a.rank() == 2) {
    Matrix* M = dynamic_cast<Matrix*>(&A);
    if (!M) dolfin_error("assembler.cpp", "assemble form", "a bilinear form needs a Matrix");
    if (M->empty()) M->init(V.pattern(keep_diagonal));
    else check_dims(*M, V);
    int i = 0;
    for (const Form::Part* p : parts) {
      if (!p) continue;
      check(db2_assemble_matrix(M->pattern(), &p->desc, p->values(), precision, M->device_values(),
                                (add_values || i > 0) ? 1 : 0, stream),
            "assemble form");
      ++i;
    }
    return;
  }
  if (a.rank() == 1) {
    Vector* b = dynamic_cast<Vector*>(&A);
    if (!b) dolfin_error("assembler.cpp", "assemble form", "a linear form needs a Vector");
    if (b->empty()) b->init(V.dim());
    else check_dims(*b, V);
    int i = 0;
    for (const Form::Part* p : parts) {
      if (!p) continue;
      check(db2_assemble_vector(V.pattern(keep_diagonal), &p->desc, p->values(), b->device_values(),
                                (add_values || i > 0) ? 1 : 0, stream),
            "assemble form");
      ++i;
    }
    return;
  }
  dolfin_error("assembler.cpp", "assemble form", "rank-0 forms are not provided by GpuAssembler");
}

GpuSystemAssembler::GpuSystemAssembler(std::shared_ptr<const Form> a, std::shared_ptr<const Form> L,
                                       std::vector<std::shared_ptr<const DirichletBC>> bcs)
    : a_(std::move(a)), L_(std::move(L)), bcs_(std::move(bcs)) {
  // SystemAssembler::check_arity (dolfin/fem/SystemAssembler.cpp)
  if (a_->rank() != 2 || L_->rank() != 1)
    dolfin_error("SystemAssembler.cpp", "assemble system", "expected a bilinear and a linear form");
  if (a_->function_space() != L_->function_space())
    dolfin_error("SystemAssembler.cpp", "assemble system", "a and L must share the function space");
  if (!a_->cell_part())
    dolfin_error("SystemAssembler.cpp", "assemble system", "the bilinear form needs a cell (dx) part");
  for (const auto& bc : bcs_)
    if (bc->function_space() != a_->function_space())
      dolfin_error("SystemAssembler.cpp", "assemble system", "boundary condition on another space");
}

void GpuSystemAssembler::assemble(Matrix& A, Vector& b) {
  const FunctionSpace& V = *a_->function_space();
  if (A.empty()) A.init(V.pattern(keep_diagonal));
  else check_dims(A, V);
  if (b.empty()) b.init(V.dim());
  else check_dims(b, V);
  const Form::Part* ac = a_->cell_part();
  const Form::Part* ads = a_->facet_part();
  const Form::Part* lds = L_->facet_part();
  // L without a dx part: the cell pass assembles a zero load
  Form::Part zero_load{make_desc(DB2_FORM_LOAD, DB2_COEFF_CONSTANT), nullptr};
  const Form::Part* lc = L_->cell_part() ? L_->cell_part() : &zero_load;
  db2_pattern P = A.pattern();
  if (!bcs_.empty()) {
    BCArrays bc;
    bc_arrays(bcs_, V.dim(), bc);
    check(db2_assemble_system_bc(P, &ac->desc, ac->values(), &lc->desc, lc->values(), bc.flags, bc.vals,
                                 precision, A.device_values(), b.device_values(), stream),
          "assemble system");
    if (ads || lds)
      check(db2_assemble_facets_bc(P, ads ? &ads->desc : nullptr, ads ? ads->values() : nullptr,
                                   lds ? &lds->desc : nullptr, lds ? lds->values() : nullptr,
                                   bc.flags, bc.vals, A.device_values(), b.device_values(), stream),
            "assemble system");
    // the flag arrays are freed when the stream has used them
    check_cuda(cudaStreamSynchronize(static_cast<cudaStream_t>(stream)), "assemble system");
    return;
  }
  check(db2_assemble_system(P, &ac->desc, ac->values(), &lc->desc, lc->values(), precision,
                            A.device_values(), b.device_values(), stream),
        "assemble system");
  if (ads)
    check(db2_assemble_matrix(P, &ads->desc, ads->values(), precision, A.device_values(), 1, stream),
          "assemble system");
  if (lds)
    check(db2_assemble_vector(P, &lds->desc, lds->values(), b.device_values(), 1, stream),
          "assemble system");
}

void GpuSystemAssembler::assemble(Matrix& A) {
  Vector b(a_->function_space()->dim());
  assemble(A, b);
}

void GpuSystemAssembler::assemble(Vector& b) {
  Matrix A;
  assemble(A, b);
}

}  // namespace dolfin_b200
