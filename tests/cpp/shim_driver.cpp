// shim_driver.cpp -- drives the C++ drop-in classes (GpuAssembler,
// GpuSystemAssembler) through include/dolfin_b200_assembler.h for the GPU
// test tests/test_gpu_cpp_shim.py, which compares what it writes with the
// Python path on the same inputs.
//
//   shim_driver <n> <input dir> <output dir>
//
// Inputs (raw little-endian doubles): coords.bin (jittered UnitCubeMesh(n)
// coordinates), kappa.bin and f.bin (P1 vertex values).  Outputs: one raw
// file per array, named <case>_<array>.bin, and error.txt.
#include <cstdio>
#include <cstdlib>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/dolfin_b200_assembler.h"

using namespace dolfin_b200;

static std::vector<double> read_doubles(const std::string& path) {
  FILE* f = std::fopen(path.c_str(), "rb");
  if (!f) throw std::runtime_error("cannot open " + path);
  std::fseek(f, 0, SEEK_END);
  const long n = std::ftell(f) / long(sizeof(double));
  std::fseek(f, 0, SEEK_SET);
  std::vector<double> v(static_cast<std::size_t>(n));
  if (std::fread(v.data(), sizeof(double), v.size(), f) != v.size()) throw std::runtime_error("short read " + path);
  std::fclose(f);
  return v;
}

template <typename T>
static void write(const std::string& path, const std::vector<T>& v) {
  FILE* f = std::fopen(path.c_str(), "wb");
  if (!f) throw std::runtime_error("cannot write " + path);
  std::fwrite(v.data(), sizeof(T), v.size(), f);
  std::fclose(f);
}

static void write_matrix(const std::string& out, const std::string& name, const Matrix& A) {
  auto d = A.data();
  write(out + "/" + name + "_rowptr.bin", std::get<0>(d));
  write(out + "/" + name + "_cols.bin", std::get<1>(d));
  write(out + "/" + name + "_vals.bin", std::get<2>(d));
}

static void write_vector(const std::string& out, const std::string& name, const Vector& b) {
  std::vector<double> x;
  b.get_local(x);
  write(out + "/" + name + "_b.bin", x);
}

int main(int argc, char** argv) {
  if (argc != 4) {
    std::fprintf(stderr, "usage: shim_driver <n> <input dir> <output dir>\n");
    return 2;
  }
  const int n = std::atoi(argv[1]);
  const std::string in = argv[2], out = argv[3];
  try {
    auto mesh = Mesh::UnitCube(n, n, n);
    mesh->set_coordinates(read_doubles(in + "/coords.bin"));
    auto P1 = std::make_shared<FunctionSpace>(mesh, 1);
    auto P2 = std::make_shared<FunctionSpace>(mesh, 2);
    auto kappa = std::make_shared<Function>(P1, read_doubles(in + "/kappa.bin"));
    auto f = std::make_shared<Function>(P1, read_doubles(in + "/f.bin"));

    // SystemAssembler(a, L).assemble(A, b): P2 kappa*grad.grad + f*v
    {
      GpuSystemAssembler S(forms::Diffusion(P2, kappa), forms::Load(P2, f));
      Matrix A;
      Vector b;
      S.assemble(A, b);
      write_matrix(out, "system", A);
      write_vector(out, "system", b);
    }
    // with ds terms and a Dirichlet condition on the face x = 0
    {
      auto a = forms::Sum(forms::Diffusion(P2, kappa), forms::BoundaryMass(P2, 0.5));
      auto L = forms::Sum(forms::Load(P2, f), forms::BoundaryLoad(P2, 1.5));
      auto bc = std::make_shared<DirichletBC>(
          P2, 0.25, [](const double* x, bool on) { return on && x[0] < 1e-12; });
      GpuSystemAssembler S(a, L, {bc});
      Matrix A;
      Vector b;
      S.assemble(A, b);
      write_matrix(out, "system_bc", A);
      write_vector(out, "system_bc", b);
    }
    // Assembler::assemble on vector P2 elasticity and its load
    {
      auto V = std::make_shared<FunctionSpace>(mesh, 2, 3);
      const double E = 1.0, nu = 0.3;
      GpuAssembler assembler;
      Matrix A;
      Vector b;
      assembler.assemble(A, *forms::Elasticity(V, E / (2 * (1 + nu)), E * nu / ((1 + nu) * (1 - 2 * nu))));
      assembler.assemble(b, *forms::Load(V, {0.0, 0.0, -1.0}));
      write_matrix(out, "elasticity", A);
      write_vector(out, "elasticity", b);
    }
    // add_values: a second assembly adds into the first
    {
      GpuAssembler assembler;
      Matrix A;
      assembler.assemble(A, *forms::Diffusion(P1, 1.7));
      assembler.add_values = true;
      assembler.assemble(A, *forms::Diffusion(P1, 1.7));
      write_matrix(out, "add_values", A);
    }
    // a tensor of the wrong size is refused with DOLFIN's message
    {
      GpuAssembler assembler;
      Vector wrong(7);
      std::string msg = "no error";
      try {
        assembler.assemble(wrong, *forms::Load(P1, f));
      } catch (const std::runtime_error& e) {
        msg = e.what();
      }
      FILE* fe = std::fopen((out + "/error.txt").c_str(), "w");
      std::fputs(msg.c_str(), fe);
      std::fclose(fe);
    }
  } catch (const std::exception& e) {
    std::fprintf(stderr, "shim_driver: %s\n", e.what());
    return 1;
  }
  return 0;
}
