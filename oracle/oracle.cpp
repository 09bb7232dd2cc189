// oracle.cpp -- CPU restatement of DOLFIN 2019.1 cell assembly.
//
// TEST INFRASTRUCTURE ONLY (the correctness checker of the CUDA engine and
// the timed CPU baseline).  The product library never links this file.
//
// Every function names the reference file:line it restates.  The element
// kernels (ufc::cell_integral::tabulate_tensor) are generated by FFC 2019.1.0
// in the reference and are not part of its source tree; they are restated
// here from the forms' definitions (exact integration of the polynomial
// integrands on affine simplices, FFC's default) with a collapsed
// Gauss--Jacobi product rule, an independent method from the engine's
// closed-form barycentric contractions.
//
// Build: see oracle/Makefile (g++ -O2 -shared -fPIC, single threaded, as the
// reference's serial assembler).

#include "oracle.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <deque>
#include <memory>
#include <numeric>
#include <stdexcept>
#include <vector>

namespace {

// --------------------------------------------------------------------------
// Reference-cell conventions (UFC).  Local edges of a cell as created by
// TetrahedronCell::create_entities (dolfin/mesh/TetrahedronCell.cpp:119-124)
// and TriangleCell::create_entities (dolfin/mesh/TriangleCell.cpp:106-108).
const int kTetEdges[6][2] = {{2, 3}, {1, 3}, {1, 2}, {0, 3}, {0, 2}, {0, 1}};
const int kTriEdges[3][2] = {{1, 2}, {0, 2}, {0, 1}};

int num_edges(int tdim) { return tdim == 3 ? 6 : (tdim == 2 ? 3 : 0); }
const int (*edge_table(int tdim))[2] { return tdim == 3 ? kTetEdges : kTriEdges; }

// Scalar Lagrange element dimension on a simplex of dimension tdim.
int scalar_dim(int family, int degree, int tdim) {
  if (family == ORC_DG && degree == 0) return 1;
  if (degree == 1) return tdim + 1;
  if (degree == 2) return (tdim + 1) + num_edges(tdim);
  return -1;
}

// --------------------------------------------------------------------------
// Gauss--Jacobi rules on [0,1] for the weight (1-u)^alpha (beta = 0), by
// Newton iteration with deflation on the Jacobi polynomial P_m^(alpha,0),
// using the three-term recurrence and P'_n = (n+a+b+1)/2 P_{n-1}^(a+1,b+1).
double jacobi(int n, double a, double b, double x) {
  if (n == 0) return 1.0;
  double p0 = 1.0;
  double p1 = 0.5 * (a - b + (a + b + 2.0) * x);
  for (int k = 2; k <= n; ++k) {
    const double c = 2.0 * k + a + b;
    const double a1 = 2.0 * k * (k + a + b) * (c - 2.0);
    const double a2 = (c - 1.0) * (a * a - b * b);
    const double a3 = (c - 2.0) * (c - 1.0) * c;
    const double a4 = 2.0 * (k + a - 1.0) * (k + b - 1.0) * c;
    const double p2 = ((a2 + a3 * x) * p1 - a4 * p0) / a1;
    p0 = p1;
    p1 = p2;
  }
  return p1;
}

double djacobi(int n, double a, double b, double x) {
  if (n == 0) return 0.0;
  return 0.5 * (n + a + b + 1.0) * jacobi(n - 1, a + 1.0, b + 1.0, x);
}

void gauss_jacobi01(int m, double alpha, std::vector<double>& u, std::vector<double>& w) {
  const double beta = 0.0;
  std::vector<double> x(m);
  for (int k = 0; k < m; ++k) {
    double r = -std::cos((2.0 * k + 1.0) * M_PI / (2.0 * m));
    for (int it = 0; it < 100; ++it) {
      const double f = jacobi(m, alpha, beta, r);
      const double df = djacobi(m, alpha, beta, r);
      double s = 0.0;
      for (int j = 0; j < k; ++j) s += 1.0 / (r - x[j]);
      const double delta = f / (df - s * f);
      r -= delta;
      if (std::fabs(delta) < 1e-16) break;
    }
    x[k] = r;
  }
  std::sort(x.begin(), x.end());
  const double lc = (alpha + beta + 1.0) * std::log(2.0) + std::lgamma(m + alpha + 1.0) +
                    std::lgamma(m + beta + 1.0) - std::lgamma(m + alpha + beta + 1.0) -
                    std::lgamma(m + 1.0);
  const double c = std::exp(lc);
  u.resize(m);
  w.resize(m);
  for (int k = 0; k < m; ++k) {
    const double d = djacobi(m, alpha, beta, x[k]);
    const double wx = c / ((1.0 - x[k] * x[k]) * d * d);
    u[k] = 0.5 * (1.0 + x[k]);
    w[k] = wx / std::pow(2.0, alpha + 1.0);
  }
}

// Collapsed (Duffy) product rule on the reference simplex, exact for
// polynomials of total degree `degree`.
struct Quadrature {
  int tdim = 0;
  std::vector<double> X;  // npts * tdim
  std::vector<double> w;  // weights summing to 1/tdim!
  int size() const { return (int)w.size(); }
};

Quadrature make_quadrature(int tdim, int degree) {
  const int m = std::max(1, (degree + 2) / 2);
  Quadrature q;
  q.tdim = tdim;
  if (tdim == 1) {
    std::vector<double> u, w;
    gauss_jacobi01(m, 0.0, u, w);
    for (int i = 0; i < m; ++i) { q.X.push_back(u[i]); q.w.push_back(w[i]); }
  } else if (tdim == 2) {
    std::vector<double> u0, w0, u1, w1;
    gauss_jacobi01(m, 1.0, u0, w0);
    gauss_jacobi01(m, 0.0, u1, w1);
    for (int i = 0; i < m; ++i)
      for (int j = 0; j < m; ++j) {
        q.X.push_back(u0[i]);
        q.X.push_back((1.0 - u0[i]) * u1[j]);
        q.w.push_back(w0[i] * w1[j]);
      }
  } else {
    std::vector<double> u0, w0, u1, w1, u2, w2;
    gauss_jacobi01(m, 2.0, u0, w0);
    gauss_jacobi01(m, 1.0, u1, w1);
    gauss_jacobi01(m, 0.0, u2, w2);
    for (int i = 0; i < m; ++i)
      for (int j = 0; j < m; ++j)
        for (int k = 0; k < m; ++k) {
          q.X.push_back(u0[i]);
          q.X.push_back((1.0 - u0[i]) * u1[j]);
          q.X.push_back((1.0 - u0[i]) * (1.0 - u1[j]) * u2[k]);
          q.w.push_back(w0[i] * w1[j] * w2[k]);
        }
  }
  return q;
}

// --------------------------------------------------------------------------
// Scalar Lagrange basis on the reference simplex.  Barycentric coordinates
// lambda_0 = 1 - sum X, lambda_{m+1} = X_m.  P1: lambda_a.  P2 (UFC order):
// vertices lambda_a (2 lambda_a - 1), then edge e = (p,q) of the local edge
// table: 4 lambda_p lambda_q.  Values and reference gradients d/dX_m.
void eval_basis(int family, int degree, int tdim, const double* X, double* phi,
                double* dphi /* ndofs * tdim */) {
  double lam[4];
  lam[0] = 1.0;
  for (int m = 0; m < tdim; ++m) { lam[m + 1] = X[m]; lam[0] -= X[m]; }
  // d lambda_a / d X_m
  auto dlam = [](int a, int m) { return a == 0 ? -1.0 : (a == m + 1 ? 1.0 : 0.0); };
  if (family == ORC_DG && degree == 0) {
    phi[0] = 1.0;
    for (int m = 0; m < tdim; ++m) dphi[m] = 0.0;
    return;
  }
  const int nv = tdim + 1;
  if (degree == 1) {
    for (int a = 0; a < nv; ++a) {
      phi[a] = lam[a];
      for (int m = 0; m < tdim; ++m) dphi[a * tdim + m] = dlam(a, m);
    }
    return;
  }
  // degree 2
  for (int a = 0; a < nv; ++a) {
    phi[a] = lam[a] * (2.0 * lam[a] - 1.0);
    for (int m = 0; m < tdim; ++m) dphi[a * tdim + m] = (4.0 * lam[a] - 1.0) * dlam(a, m);
  }
  const int ne = num_edges(tdim);
  const int (*E)[2] = edge_table(tdim);
  if (tdim == 1) return;
  for (int e = 0; e < ne; ++e) {
    const int p = E[e][0], q = E[e][1];
    phi[nv + e] = 4.0 * lam[p] * lam[q];
    for (int m = 0; m < tdim; ++m)
      dphi[(nv + e) * tdim + m] = 4.0 * (dlam(p, m) * lam[q] + lam[p] * dlam(q, m));
  }
}

int coeff_degree(int coeff) {
  switch (coeff) {
    case ORC_COEFF_P1: case ORC_COEFF_X0: return 1;
    case ORC_COEFF_P1_TIMES_P1: return 2;
    default: return 0;
  }
}

int form_rank(int kind) {
  switch (kind) {
    case ORC_LOAD: case ORC_FACET_LOAD: return 1;
    case ORC_FUNCTIONAL: case ORC_FACET_FUNCTIONAL: return 0;
    default: return 2;
  }
}

bool is_facet_kind(int kind) {
  return kind == ORC_FACET_MASS || kind == ORC_FACET_LOAD || kind == ORC_FACET_FUNCTIONAL;
}

int quadrature_degree(const orc_form& f) {
  const int c = coeff_degree(f.coeff);
  const int p0 = f.degree0, p1 = f.degree1;
  switch (f.kind) {
    case ORC_DIFFUSION: return 2 * std::max(p0, p1) - 2 + c;
    case ORC_MASS: return p0 + p1 + c;
    case ORC_LOAD: return p0 + c;
    case ORC_ELASTICITY: return p0 + p1 - 2;
    case ORC_DIV_P: return p0 - 1 + p1;
    case ORC_GRADP_V: return p0 + p1 - 1;
    case ORC_FACET_MASS: return p0 + p1 + c;
    case ORC_FACET_LOAD: return p0 + c;
    default: return c;
  }
}

// Per-form tabulation context: quadrature + basis tables at the points
// (computed once, as FFC-generated code tabulates them at compile time).
struct Tabulator {
  orc_form f;
  Quadrature q;
  int k0 = 0, k1 = 0;  // scalar element dims
  int n0 = 0, n1 = 0;  // element tensor dims (k * vsize)
  std::vector<double> phi0, dphi0, phi1, dphi1, lam;

  explicit Tabulator(const orc_form& form) : f(form) {
    const int d = f.tdim;
    q = make_quadrature(d, quadrature_degree(f));
    const int rank = form_rank(f.kind);
    if (rank >= 1) {
      k0 = scalar_dim(f.family0, f.degree0, d);
      n0 = k0 * f.vsize0;
    }
    if (rank == 2) {
      k1 = scalar_dim(f.family1, f.degree1, d);
      n1 = k1 * f.vsize1;
    }
    const int np = q.size();
    phi0.resize(np * std::max(k0, 1));
    dphi0.resize(np * std::max(k0, 1) * d);
    phi1.resize(np * std::max(k1, 1));
    dphi1.resize(np * std::max(k1, 1) * d);
    lam.resize(np * (d + 1));
    for (int p = 0; p < np; ++p) {
      const double* X = &q.X[p * d];
      if (k0) eval_basis(f.family0, f.degree0, d, X, &phi0[p * k0], &dphi0[p * k0 * d]);
      if (k1) eval_basis(f.family1, f.degree1, d, X, &phi1[p * k1], &dphi1[p * k1 * d]);
      double s = 0.0;
      for (int m = 0; m < d; ++m) { lam[p * (d + 1) + m + 1] = X[m]; s += X[m]; }
      lam[p * (d + 1)] = 1.0 - s;
    }
  }

  // Affine geometry: J[r][m] = x_{m+1}[r] - x_0[r]; returns det, fills Kinv = J^{-1}.
  static double geometry(int d, const double* xc, double* Kinv) {
    double J[3][3];
    for (int r = 0; r < d; ++r)
      for (int m = 0; m < d; ++m) J[r][m] = xc[(m + 1) * d + r] - xc[r];
    double det;
    if (d == 1) {
      det = J[0][0];
      Kinv[0] = 1.0 / det;
    } else if (d == 2) {
      det = J[0][0] * J[1][1] - J[0][1] * J[1][0];
      Kinv[0] = J[1][1] / det;
      Kinv[1] = -J[0][1] / det;
      Kinv[2] = -J[1][0] / det;
      Kinv[3] = J[0][0] / det;
    } else {
      const double c00 = J[1][1] * J[2][2] - J[1][2] * J[2][1];
      const double c01 = J[1][2] * J[2][0] - J[1][0] * J[2][2];
      const double c02 = J[1][0] * J[2][1] - J[1][1] * J[2][0];
      det = J[0][0] * c00 + J[0][1] * c01 + J[0][2] * c02;
      // inverse = adjugate / det; adj[m][r] = cofactor[r][m]
      Kinv[0 * 3 + 0] = c00 / det;
      Kinv[1 * 3 + 0] = c01 / det;
      Kinv[2 * 3 + 0] = c02 / det;
      Kinv[0 * 3 + 1] = (J[0][2] * J[2][1] - J[0][1] * J[2][2]) / det;
      Kinv[1 * 3 + 1] = (J[0][0] * J[2][2] - J[0][2] * J[2][0]) / det;
      Kinv[2 * 3 + 1] = (J[0][1] * J[2][0] - J[0][0] * J[2][1]) / det;
      Kinv[0 * 3 + 2] = (J[0][1] * J[1][2] - J[0][2] * J[1][1]) / det;
      Kinv[1 * 3 + 2] = (J[0][2] * J[1][0] - J[0][0] * J[1][2]) / det;
      Kinv[2 * 3 + 2] = (J[0][0] * J[1][1] - J[0][1] * J[1][0]) / det;
    }
    return det;
  }

  double coeff_at(int p, const double* xc, const double* w, const double* w2) const {
    const int d = f.tdim;
    const double* l = &lam[p * (d + 1)];
    switch (f.coeff) {
      case ORC_COEFF_CONST: return f.c[0];
      case ORC_COEFF_P1: {
        double s = 0.0;
        for (int a = 0; a <= d; ++a) s += w[a] * l[a];
        return s;
      }
      case ORC_COEFF_X0: {
        const int comp = (int)f.c[1];
        double s = 0.0;
        for (int a = 0; a <= d; ++a) s += xc[a * d + comp] * l[a];
        return s;
      }
      case ORC_COEFF_P1_TIMES_P1: {
        double s = 0.0, s2 = 0.0;
        for (int a = 0; a <= d; ++a) { s += w[a] * l[a]; s2 += w2[a] * l[a]; }
        return s * s2;
      }
      default: return 1.0;
    }
  }

  // tabulate_tensor: A row-major over (test, trial); A must hold n0*n1
  // (rank 2), n0 (rank 1) or 1 (rank 0) values.
  void tabulate(const double* xc, const double* w, const double* w2, double* A) const {
    const int d = f.tdim;
    const int rank = form_rank(f.kind);
    const int size = rank == 2 ? n0 * n1 : (rank == 1 ? n0 : 1);
    std::fill(A, A + size, 0.0);
    double Kinv[9];
    const double det = geometry(d, xc, Kinv);
    const double adet = std::fabs(det);
    double G0[30 * 3], G1[30 * 3];
    for (int p = 0; p < q.size(); ++p) {
      const double wq = q.w[p] * adet;
      const double kq = coeff_at(p, xc, w, w2);
      // physical gradients: G[i][r] = sum_m Kinv[m][r] dphi[i][m]
      for (int i = 0; i < k0; ++i)
        for (int r = 0; r < d; ++r) {
          double s = 0.0;
          for (int m = 0; m < d; ++m) s += Kinv[m * d + r] * dphi0[(p * k0 + i) * d + m];
          G0[i * d + r] = s;
        }
      for (int j = 0; j < k1; ++j)
        for (int r = 0; r < d; ++r) {
          double s = 0.0;
          for (int m = 0; m < d; ++m) s += Kinv[m * d + r] * dphi1[(p * k1 + j) * d + m];
          G1[j * d + r] = s;
        }
      const double* ph0 = &phi0[p * std::max(k0, 1)];
      const double* ph1 = &phi1[p * std::max(k1, 1)];
      switch (f.kind) {
        case ORC_DIFFUSION:
          for (int i = 0; i < k0; ++i)
            for (int j = 0; j < k1; ++j) {
              double g = 0.0;
              for (int r = 0; r < d; ++r) g += G0[i * d + r] * G1[j * d + r];
              A[i * n1 + j] += wq * kq * g;
            }
          break;
        case ORC_MASS:
          for (int i = 0; i < k0; ++i)
            for (int j = 0; j < k1; ++j) A[i * n1 + j] += wq * kq * ph0[i] * ph1[j];
          break;
        case ORC_LOAD:
          if (f.vsize0 == 1) {
            for (int i = 0; i < k0; ++i) A[i] += wq * kq * ph0[i];
          } else {
            for (int c = 0; c < f.vsize0; ++c)
              for (int i = 0; i < k0; ++i) A[c * k0 + i] += wq * f.c[c] * ph0[i];
          }
          break;
        case ORC_ELASTICITY:
          for (int c = 0; c < f.vsize0; ++c)
            for (int i = 0; i < k0; ++i)
              for (int e = 0; e < f.vsize1; ++e)
                for (int j = 0; j < k1; ++j) {
                  double g = 0.0;
                  for (int r = 0; r < d; ++r) g += G0[i * d + r] * G1[j * d + r];
                  const double v = f.lmbda * G0[i * d + c] * G1[j * d + e] +
                                   f.mu * ((c == e ? g : 0.0) + G0[i * d + e] * G1[j * d + c]);
                  A[(c * k0 + i) * n1 + e * k1 + j] += wq * v;
                }
          break;
        case ORC_DIV_P:
          for (int c = 0; c < f.vsize0; ++c)
            for (int i = 0; i < k0; ++i)
              for (int j = 0; j < k1; ++j) A[(c * k0 + i) * n1 + j] += wq * G0[i * d + c] * ph1[j];
          break;
        case ORC_GRADP_V:
          for (int c = 0; c < f.vsize0; ++c)
            for (int i = 0; i < k0; ++i)
              for (int j = 0; j < k1; ++j) A[(c * k0 + i) * n1 + j] += wq * ph0[i] * G1[j * d + c];
          break;
        case ORC_FUNCTIONAL:
          A[0] += wq * kq;
          break;
        default:
          throw std::runtime_error("unknown form");
      }
    }
  }
};

// Exterior facet integrals (ufc::exterior_facet_integral::tabulate_tensor,
// FFC-generated; called at Assembler.cpp:277-281): the facet tensor in the
// cell's local dof layout, integrated exactly with a Gauss--Jacobi rule on the
// reference facet mapped into the cell.  Local facet f is opposite local
// vertex f; its points have cell barycentrics lambda_f = 0 and lambda_{a_k} =
// mu_k for the facet's vertices a_0 < a_1 (< a_2).  The physical measure is
// |F| (d-1)! times the reference facet weight.
struct FacetTabulator {
  orc_form f;
  Quadrature q;
  int k0 = 0, k1 = 0, n0 = 0, n1 = 0;
  // per local facet: basis values and cell barycentrics at the points
  std::vector<double> phi0[4], phi1[4], lam[4];

  explicit FacetTabulator(const orc_form& form) : f(form) {
    const int d = f.tdim;
    q = make_quadrature(d - 1, quadrature_degree(f));
    const int rank = form_rank(f.kind);
    if (rank >= 1) { k0 = scalar_dim(f.family0, f.degree0, d); n0 = k0 * f.vsize0; }
    if (rank == 2) { k1 = scalar_dim(f.family1, f.degree1, d); n1 = k1 * f.vsize1; }
    const int np = q.size();
    std::vector<double> dummy(30 * 3);
    for (int fl = 0; fl <= d; ++fl) {
      int av[3], m = 0;
      for (int a = 0; a <= d; ++a)
        if (a != fl) av[m++] = a;
      phi0[fl].resize(np * std::max(k0, 1));
      phi1[fl].resize(np * std::max(k1, 1));
      lam[fl].resize(np * (d + 1));
      for (int p = 0; p < np; ++p) {
        double mu[3], s = 0.0;
        for (int r = 0; r < d - 1; ++r) { mu[r + 1] = q.X[p * (d - 1) + r]; s += mu[r + 1]; }
        mu[0] = 1.0 - s;
        double l[4] = {0, 0, 0, 0};
        for (int k = 0; k < d; ++k) l[av[k]] = mu[k];
        double X[3];
        for (int r = 0; r < d; ++r) X[r] = l[r + 1];
        for (int a = 0; a <= d; ++a) lam[fl][p * (d + 1) + a] = l[a];
        if (k0) eval_basis(f.family0, f.degree0, d, X, &phi0[fl][p * k0], dummy.data());
        if (k1) eval_basis(f.family1, f.degree1, d, X, &phi1[fl][p * k1], dummy.data());
        // basis functions of nodes off the facet (its opposite vertex, and for
        // P2 the edges through that vertex) vanish identically on it: store
        // exact zeros rather than the roundoff of lambda_0 = 1 - sum X
        for (int i = 0; i < std::max(k0, k1); ++i) {
          bool on = true;
          if (i <= d) on = i != fl;
          else {
            const int (*E)[2] = edge_table(d);
            on = E[i - d - 1][0] != fl && E[i - d - 1][1] != fl;
          }
          if (!on) {
            if (i < k0) phi0[fl][p * k0 + i] = 0.0;
            if (i < k1) phi1[fl][p * k1 + i] = 0.0;
          }
        }
      }
    }
  }

  // |F| (d-1)!: the facet's length (2D) or twice its area (3D)
  static double measure_factor(int d, const double* xc, int fl) {
    int av[3], m = 0;
    for (int a = 0; a <= d; ++a)
      if (a != fl) av[m++] = a;
    if (d == 2) {
      const double dx = xc[av[1] * 2] - xc[av[0] * 2], dy = xc[av[1] * 2 + 1] - xc[av[0] * 2 + 1];
      return std::sqrt(dx * dx + dy * dy);
    }
    double u[3], v[3];
    for (int r = 0; r < 3; ++r) {
      u[r] = xc[av[1] * 3 + r] - xc[av[0] * 3 + r];
      v[r] = xc[av[2] * 3 + r] - xc[av[0] * 3 + r];
    }
    const double cx = u[1] * v[2] - u[2] * v[1], cy = u[2] * v[0] - u[0] * v[2],
                 cz = u[0] * v[1] - u[1] * v[0];
    return std::sqrt(cx * cx + cy * cy + cz * cz);
  }

  void tabulate(const double* xc, const double* w, int fl, double* A) const {
    const int d = f.tdim;
    const int rank = form_rank(f.kind);
    const int size = rank == 2 ? n0 * n1 : (rank == 1 ? n0 : 1);
    std::fill(A, A + size, 0.0);
    const double scale = measure_factor(d, xc, fl);
    for (int p = 0; p < q.size(); ++p) {
      const double* l = &lam[fl][p * (d + 1)];
      double kq = 1.0;
      if (f.coeff == ORC_COEFF_CONST) kq = f.c[0];
      else if (f.coeff == ORC_COEFF_P1) {
        kq = 0.0;
        for (int a = 0; a <= d; ++a) kq += w[a] * l[a];
      } else if (f.coeff == ORC_COEFF_X0) {
        const int comp = (int)f.c[1];
        kq = 0.0;
        for (int a = 0; a <= d; ++a) kq += xc[a * d + comp] * l[a];
      }
      const double wq = q.w[p] * scale;
      const double* ph0 = &phi0[fl][p * std::max(k0, 1)];
      const double* ph1 = &phi1[fl][p * std::max(k1, 1)];
      switch (f.kind) {
        case ORC_FACET_MASS:
          for (int i = 0; i < k0; ++i)
            for (int j = 0; j < k1; ++j) A[i * n1 + j] += wq * kq * ph0[i] * ph1[j];
          break;
        case ORC_FACET_LOAD:
          if (f.vsize0 == 1) {
            for (int i = 0; i < k0; ++i) A[i] += wq * kq * ph0[i];
          } else {
            for (int c = 0; c < f.vsize0; ++c)
              for (int i = 0; i < k0; ++i) A[c * k0 + i] += wq * f.c[c] * ph0[i];
          }
          break;
        case ORC_FACET_FUNCTIONAL:
          A[0] += wq * kq;
          break;
        default:
          throw std::runtime_error("not a facet form");
      }
    }
  }
};

// Facet::exterior() (one incident cell) over the facets numbered by
// TopologyComputation::compute_entities_by_key_matching
// (dolfin/mesh/TopologyComputation.cpp:152-330): sorted vertex keys, in key
// order.  Cell facet i is opposite local vertex i
// (TetrahedronCell::create_entities / TriangleCell::create_entities).
struct ExtFacets {
  std::vector<uint32_t> cell;
  std::vector<int32_t> local;
};

ExtFacets exterior_facets(int d, int64_t nc, const uint32_t* cells) {
  struct Keyed { uint32_t k[3]; int64_t slot; };
  const int nf = d + 1;
  std::vector<Keyed> keyed((size_t)nc * nf);
  for (int64_t c = 0; c < nc; ++c)
    for (int fl = 0; fl < nf; ++fl) {
      Keyed& K = keyed[c * nf + fl];
      int m = 0;
      for (int a = 0; a <= d; ++a)
        if (a != fl) K.k[m++] = cells[c * nf + a];
      for (; m < 3; ++m) K.k[m] = 0;
      std::sort(K.k, K.k + d);
      K.slot = c * nf + fl;
    }
  auto less = [](const Keyed& x, const Keyed& y) {
    for (int r = 0; r < 3; ++r)
      if (x.k[r] != y.k[r]) return x.k[r] < y.k[r];
    return x.slot < y.slot;
  };
  std::sort(keyed.begin(), keyed.end(), less);
  ExtFacets E;
  size_t i = 0;
  while (i < keyed.size()) {
    size_t j = i + 1;
    while (j < keyed.size() && std::equal(keyed[j].k, keyed[j].k + 3, keyed[i].k)) ++j;
    if (j - i == 1) {
      E.cell.push_back((uint32_t)(keyed[i].slot / nf));
      E.local.push_back((int32_t)(keyed[i].slot % nf));
    }
    i = j;
  }
  return E;
}

// Cell::get_coordinate_dofs (dolfin/mesh/Cell.h:293-307): vertex-major copy.
void gather_coordinates(int d, const double* coords, const uint32_t* cell, double* xc) {
  for (int a = 0; a <= d; ++a)
    for (int r = 0; r < d; ++r) xc[a * d + r] = coords[(int64_t)cell[a] * d + r];
}

// Function::restrict for a P1 field (dolfin/function/Function.cpp:449-469):
// the cell's vertex values (P1 dof == vertex index under natural numbering).
void gather_vertex_field(int d, const double* w, const uint32_t* cell, double* wc) {
  for (int a = 0; a <= d; ++a) wc[a] = w ? w[cell[a]] : 0.0;
}

// EigenMatrix::add (dolfin/la/EigenMatrix.cpp:156-166): coeffRef(row,col) +=
// on a compressed row-major matrix, i.e. a binary search inside the row.
inline bool csr_add(const int32_t* rowptr, const int32_t* cols, double* vals, int32_t row,
                    int32_t col, double v) {
  const int32_t* b = cols + rowptr[row];
  const int32_t* e = cols + rowptr[row + 1];
  const int32_t* it = std::lower_bound(b, e, col);
  if (it == e || *it != col) return false;
  vals[it - cols] += v;
  return true;
}

struct CSR {
  std::vector<int32_t> rowptr, cols;
};

}  // namespace

struct orc_csr {
  CSR csr;
};

extern "C" {

// BoxMesh::build_tet (dolfin/generation/BoxMesh.cpp:50-170) on the unit cube,
// followed by MeshEditor::close -> TetrahedronCell::order (cell vertices
// sorted ascending, dolfin/mesh/TetrahedronCell.cpp:455).
int orc_box_mesh(int nx, int ny, int nz, double* coords, uint32_t* cells) {
  if (nx < 1 || ny < 1 || nz < 1) return -1;
  const double a = 0.0, b = 1.0, c = 0.0, d = 1.0, e = 0.0, f = 1.0;
  int64_t v = 0;
  for (int iz = 0; iz <= nz; ++iz) {
    const double z = e + (static_cast<double>(iz)) * (f - e) / static_cast<double>(nz);
    for (int iy = 0; iy <= ny; ++iy) {
      const double y = c + (static_cast<double>(iy)) * (d - c) / static_cast<double>(ny);
      for (int ix = 0; ix <= nx; ++ix) {
        const double x = a + (static_cast<double>(ix)) * (b - a) / static_cast<double>(nx);
        coords[3 * v + 0] = x;
        coords[3 * v + 1] = y;
        coords[3 * v + 2] = z;
        ++v;
      }
    }
  }
  int64_t cell = 0;
  for (int iz = 0; iz < nz; ++iz)
    for (int iy = 0; iy < ny; ++iy)
      for (int ix = 0; ix < nx; ++ix) {
        const uint32_t v0 = iz * (nx + 1) * (ny + 1) + iy * (nx + 1) + ix;
        const uint32_t v1 = v0 + 1;
        const uint32_t v2 = v0 + (nx + 1);
        const uint32_t v3 = v1 + (nx + 1);
        const uint32_t v4 = v0 + (nx + 1) * (ny + 1);
        const uint32_t v5 = v1 + (nx + 1) * (ny + 1);
        const uint32_t v6 = v2 + (nx + 1) * (ny + 1);
        const uint32_t v7 = v3 + (nx + 1) * (ny + 1);
        const uint32_t lists[6][4] = {{v0, v1, v3, v7}, {v0, v1, v7, v5}, {v0, v5, v7, v4},
                                      {v0, v3, v2, v7}, {v0, v6, v4, v7}, {v0, v2, v6, v7}};
        for (int t = 0; t < 6; ++t) {
          uint32_t* out = cells + 4 * cell;
          std::copy(lists[t], lists[t] + 4, out);
          std::sort(out, out + 4);
          ++cell;
        }
      }
  return 0;
}

// RectangleMesh::build_tri (dolfin/generation/RectangleMesh.cpp:46-233) on
// the unit square (UnitSquareMesh, default diagonal "right").
int orc_rectangle_mesh(int nx, int ny, int diagonal, double* coords, uint32_t* cells) {
  if (nx < 1 || ny < 1) return -1;
  const double a = 0.0, b = 1.0, c = 0.0, d = 1.0;
  int64_t v = 0;
  for (int iy = 0; iy <= ny; ++iy) {
    const double y = c + ((static_cast<double>(iy)) * (d - c) / static_cast<double>(ny));
    for (int ix = 0; ix <= nx; ++ix) {
      const double x = a + ((static_cast<double>(ix)) * (b - a) / static_cast<double>(nx));
      coords[2 * v + 0] = x;
      coords[2 * v + 1] = y;
      ++v;
    }
  }
  int64_t cell = 0;
  for (int iy = 0; iy < ny; ++iy) {
    // diagonal 0 right, 1 left, 2 right/left, 3 left/right
    bool left;
    if (diagonal == 2) left = !(iy % 2);
    else if (diagonal == 3) left = (iy % 2);
    else left = (diagonal == 1);
    for (int ix = 0; ix < nx; ++ix) {
      const uint32_t v0 = iy * (nx + 1) + ix;
      const uint32_t v1 = v0 + 1;
      const uint32_t v2 = v0 + (nx + 1);
      const uint32_t v3 = v1 + (nx + 1);
      uint32_t c0[3], c1[3];
      if (left) {
        c0[0] = v0; c0[1] = v1; c0[2] = v2;
        c1[0] = v1; c1[1] = v2; c1[2] = v3;
      } else {
        c0[0] = v0; c0[1] = v1; c0[2] = v3;
        c1[0] = v0; c1[1] = v2; c1[2] = v3;
      }
      if (diagonal >= 2) left = !left;
      for (const uint32_t* src : {c0, c1}) {
        uint32_t* out = cells + 3 * cell;
        std::copy(src, src + 3, out);
        std::sort(out, out + 3);
        ++cell;
      }
    }
  }
  return 0;
}

// IntervalMesh (dolfin/generation/IntervalMesh.cpp) on [0,1].
int orc_interval_mesh(int n, double* coords, uint32_t* cells) {
  if (n < 1) return -1;
  for (int i = 0; i <= n; ++i) coords[i] = 0.0 + static_cast<double>(i) * (1.0 - 0.0) / static_cast<double>(n);
  for (int i = 0; i < n; ++i) { cells[2 * i] = i; cells[2 * i + 1] = i + 1; }
  return 0;
}

// TopologyComputation::compute_entities_by_key_matching
// (dolfin/mesh/TopologyComputation.cpp:152-330): entities are keyed by their
// sorted vertex tuple, sorted, and numbered in key order.
int64_t orc_edges(int tdim, int64_t nc, const uint32_t* cells, uint32_t* cell_edges,
                  uint32_t* edge_vertices) {
  const int ne = num_edges(tdim);
  const int nv = tdim + 1;
  if (ne == 0) return 0;
  const int (*E)[2] = edge_table(tdim);
  struct Keyed { uint64_t key; int64_t slot; };
  std::vector<Keyed> keyed((size_t)nc * ne);
  for (int64_t c = 0; c < nc; ++c)
    for (int i = 0; i < ne; ++i) {
      uint32_t p = cells[c * nv + E[i][0]], q = cells[c * nv + E[i][1]];
      if (p > q) std::swap(p, q);
      keyed[c * ne + i] = {((uint64_t)p << 32) | q, c * ne + i};
    }
  std::sort(keyed.begin(), keyed.end(), [](const Keyed& x, const Keyed& y) {
    return x.key < y.key || (x.key == y.key && x.slot < y.slot);
  });
  int64_t index = -1;
  uint64_t prev = ~(uint64_t)0;
  for (const auto& k : keyed) {
    if (k.key != prev) {
      ++index;
      prev = k.key;
      if (edge_vertices) {
        edge_vertices[2 * index] = (uint32_t)(k.key >> 32);
        edge_vertices[2 * index + 1] = (uint32_t)(k.key & 0xffffffffu);
      }
    }
    cell_edges[k.slot] = (uint32_t)index;
  }
  return index + 1;
}

int orc_ndofs_per_cell(int family, int degree, int vsize, int tdim) {
  return scalar_dim(family, degree, tdim) * vsize;
}

// DofMapBuilder::build with reorder_dofs_serial = false
// (dolfin/fem/DofMapBuilder.cpp:253-272): the UFC tabulate_dofs numbering
// (build_ufc_node_graph, :1127-1154).  Lagrange: vertex dofs first, then
// Nv + edge index; vector elements component-major, component c offset by
// c * (scalar global dimension).  DG: cell-interior numbering.
int64_t orc_dofmap(int family, int degree, int vsize, int tdim, int64_t nv, int64_t nc,
                   const uint32_t* cells, int32_t* cell_dofs) {
  const int k = scalar_dim(family, degree, tdim);
  if (k <= 0) return -1;
  const int nvc = tdim + 1;
  std::vector<uint32_t> cedges;
  int64_t ne = 0;
  if (family == ORC_CG && degree == 2) {
    cedges.resize((size_t)nc * num_edges(tdim));
    ne = orc_edges(tdim, nc, cells, cedges.data(), nullptr);
  }
  int64_t nscalar;
  if (family == ORC_DG) nscalar = nc * k;
  else nscalar = nv + (degree == 2 ? ne : 0);
  const int n = k * vsize;
  for (int64_t c = 0; c < nc; ++c) {
    int32_t sd[16];
    if (family == ORC_DG) {
      for (int i = 0; i < k; ++i) sd[i] = (int32_t)(c * k + i);
    } else {
      for (int a = 0; a < nvc; ++a) sd[a] = (int32_t)cells[c * nvc + a];
      if (degree == 2)
        for (int e = 0; e < num_edges(tdim); ++e)
          sd[nvc + e] = (int32_t)(nv + cedges[c * num_edges(tdim) + e]);
    }
    for (int comp = 0; comp < vsize; ++comp)
      for (int i = 0; i < k; ++i) cell_dofs[c * n + comp * k + i] = (int32_t)(comp * nscalar + sd[i]);
  }
  return nscalar * vsize;
}

// ---- reordered dofmap -------------------------------------------------------
// DofMapBuilder::compute_node_reordering (dolfin/fem/DofMapBuilder.cpp:
// 1473-1667) on one process: graph[n0].insert(n1) for every ordered pair of
// distinct nodes of every cell (dolfin::Set, dolfin/common/Set.h:79-96), then
// BoostGraphOrdering::compute_cuthill_mckee(graph, true)
// (dolfin/graph/BoostGraphOrdering.cpp:34-75), then build_dofmap (:1669-1693):
// dof = bs*new_node + component.  The Boost algorithm (not in the reference
// tree) is restated after boost/graph/cuthill_mckee_ordering.hpp and
// sparse_ordering.hpp: rcm_queue-style level bookkeeping for the
// pseudo-peripheral search, and a BFS whose visitor sorts the vertices it
// enqueued for each examined vertex by degree.
namespace {

struct LevelQueue {  // Boost's rcm_queue
  std::deque<int32_t> q;
  const std::vector<int32_t>* deg;
  size_t in_level = 0, level_size = 1;
  int ecc = -1;
  int32_t spouse = -1;
  int32_t front() {
    const int32_t u = q.front();
    if (in_level == 0) spouse = u;
    else if ((*deg)[u] < (*deg)[spouse]) spouse = u;
    return u;
  }
  void pop() {
    if (!in_level) level_size = q.size();
    q.pop_front();
    if (in_level == level_size - 1) {
      in_level = 0;
      ++ecc;
    } else {
      ++in_level;
    }
  }
};

int32_t peripheral_pair(const std::vector<std::vector<int32_t>>& g, const std::vector<int32_t>& deg,
                        int32_t u, int& ecc) {
  std::vector<uint8_t> seen(g.size(), 0);
  LevelQueue Q;
  Q.deg = &deg;
  Q.q.push_back(u);
  seen[u] = 1;
  while (!Q.q.empty()) {
    const int32_t x = Q.front();
    Q.pop();
    for (int32_t y : g[x])
      if (!seen[y]) {
        seen[y] = 1;
        Q.q.push_back(y);
      }
  }
  ecc = Q.ecc;
  return Q.spouse;
}

std::vector<int32_t> boost_rcm(const std::vector<std::vector<int32_t>>& g) {
  const int32_t n = (int32_t)g.size();
  std::vector<int32_t> deg(n);
  for (int32_t v = 0; v < n; ++v) deg[v] = (int32_t)g[v].size();
  std::vector<int32_t> map(n);
  bool any = false;
  for (int32_t v = 0; v < n; ++v) any |= !g[v].empty();
  if (!any) {
    for (int32_t v = 0; v < n; ++v) map[v] = v;
    return map;
  }
  // one vertex per component, in vertex order (depth_first_visit from each
  // still-white vertex)
  std::vector<uint8_t> col(n, 0);
  std::vector<int32_t> comp;
  for (int32_t v = 0; v < n; ++v) {
    if (col[v]) continue;
    comp.push_back(v);
    std::vector<int32_t> st{v};
    col[v] = 1;
    while (!st.empty()) {
      const int32_t u = st.back();
      st.pop_back();
      for (int32_t w : g[u])
        if (!col[w]) { col[w] = 1; st.push_back(w); }
    }
  }
  for (int32_t& r : comp) {  // find_starting_node
    int er, ex;
    int32_t x = peripheral_pair(g, deg, r, er);
    int32_t y = peripheral_pair(g, deg, x, ex);
    while (ex > er) {
      r = x;
      er = ex;
      x = y;
      y = peripheral_pair(g, deg, x, ex);
    }
    r = x;
  }
  std::vector<uint8_t> color(n, 0);  // white 0, gray 1, black 2
  std::vector<int32_t> perm;         // visit order
  std::deque<int32_t> Q;
  for (int32_t s : comp) {
    color[s] = 1;
    Q.push_back(s);
    while (!Q.empty()) {
      const int32_t u = Q.front();
      Q.pop_front();
      perm.push_back(u);                       // examine_vertex
      const size_t first_child = Q.size();
      for (int32_t v : g[u])
        if (color[v] == 0) { color[v] = 1; Q.push_back(v); }
      color[u] = 2;
      std::sort(Q.begin() + first_child, Q.end(),   // finish_vertex
                [&](int32_t a, int32_t b) { return deg[a] < deg[b]; });
    }
  }
  // written through inv_perm.rbegin(), then map[inv_perm[i]] = i
  for (int32_t i = 0; i < n; ++i) map[perm[i]] = n - 1 - i;
  return map;
}

}  // namespace

int64_t orc_dofmap_reordered(int degree, int vsize, int tdim, int64_t nv, int64_t nc,
                             const uint32_t* cells, int32_t* cell_dofs, int32_t* node_new) {
  const int k = scalar_dim(ORC_CG, degree, tdim);
  std::vector<int32_t> nodes((size_t)nc * k);
  const int64_t nn = orc_dofmap(ORC_CG, degree, 1, tdim, nv, nc, cells, nodes.data());
  std::vector<std::vector<int32_t>> g(nn);
  for (int64_t c = 0; c < nc; ++c)
    for (int i = 0; i < k; ++i)
      for (int j = 0; j < k; ++j) {
        if (i == j) continue;
        std::vector<int32_t>& set = g[nodes[c * k + i]];
        const int32_t x = nodes[c * k + j];
        if (std::find(set.begin(), set.end(), x) == set.end()) set.push_back(x);
      }
  const std::vector<int32_t> map = boost_rcm(g);
  for (int64_t c = 0; c < nc; ++c)
    for (int i = 0; i < k; ++i)
      for (int b = 0; b < vsize; ++b)
        cell_dofs[c * k * vsize + b * k + i] = vsize * map[nodes[c * k + i]] + b;
  if (node_new) std::copy(map.begin(), map.end(), node_new);
  return nn * vsize;
}

// SparsityPatternBuilder::build over cells (dolfin/fem/SparsityPatternBuilder.cpp:94-111)
// with SparsityPattern::insert_entries (dolfin/la/SparsityPattern.cpp:167-206,
// dolfin::Set linear-search insert, dolfin/common/Set.h:79-96), optional
// diagonal (AssemblerBase.cpp:145-163), then diagonal_pattern(sorted)
// (SparsityPattern.cpp:511-522) as inserted by EigenMatrix::init.
orc_csr* orc_sparsity(int64_t nrows, int64_t ncols, int64_t nc, int k0, const int32_t* dofs0,
                      int k1, const int32_t* dofs1, int keep_diagonal) {
  std::vector<std::vector<int32_t>> rows(nrows);
  for (int64_t c = 0; c < nc; ++c) {
    const int32_t* d0 = dofs0 + c * k0;
    const int32_t* d1 = dofs1 + c * k1;
    for (int i = 0; i < k0; ++i) {
      auto& row = rows[d0[i]];
      for (int j = 0; j < k1; ++j)
        if (std::find(row.begin(), row.end(), d1[j]) == row.end()) row.push_back(d1[j]);
    }
  }
  if (keep_diagonal) {
    const int64_t r = std::min(nrows, ncols);
    for (int64_t i = 0; i < r; ++i) {
      auto& row = rows[i];
      if (std::find(row.begin(), row.end(), (int32_t)i) == row.end()) row.push_back((int32_t)i);
    }
  }
  auto* p = new orc_csr;
  p->csr.rowptr.resize(nrows + 1);
  p->csr.rowptr[0] = 0;
  for (int64_t i = 0; i < nrows; ++i) {
    std::sort(rows[i].begin(), rows[i].end());
    p->csr.rowptr[i + 1] = p->csr.rowptr[i] + (int32_t)rows[i].size();
  }
  p->csr.cols.reserve(p->csr.rowptr[nrows]);
  for (auto& r : rows) p->csr.cols.insert(p->csr.cols.end(), r.begin(), r.end());
  return p;
}

int64_t orc_csr_nnz(const orc_csr* p) { return (int64_t)p->csr.cols.size(); }
void orc_csr_copy(const orc_csr* p, int32_t* rowptr, int32_t* cols) {
  std::copy(p->csr.rowptr.begin(), p->csr.rowptr.end(), rowptr);
  std::copy(p->csr.cols.begin(), p->csr.cols.end(), cols);
}
void orc_csr_free(orc_csr* p) { delete p; }

int orc_element_tensor(const orc_form* f, const double* coordinate_dofs, const double* w,
                       const double* w2, double* A) {
  try {
    Tabulator t(*f);
    t.tabulate(coordinate_dofs, w, w2, A);
  } catch (...) {
    return -1;
  }
  return 0;
}

// Assembler::assemble_cells (dolfin/fem/Assembler.cpp:148-193): for each cell
// in order, gather coordinates and coefficients, tabulate, and add_local into
// the matrix (EigenMatrix::add, row-major within the element).
int orc_assemble_matrix(const orc_form* f, int64_t nv, const double* coords, int64_t nc,
                        const uint32_t* cells, const int32_t* dofs0, const int32_t* dofs1,
                        const double* w, const double* w2, int64_t nrows, const int32_t* rowptr,
                        const int32_t* cols, double* vals, int add_values) {
  (void)nv;
  const int d = f->tdim;
  if (is_facet_kind(f->kind)) {
    // Assembler::assemble_exterior_facets (dolfin/fem/Assembler.cpp:196-288)
    FacetTabulator t(*f);
    if (!add_values) std::fill(vals, vals + rowptr[nrows], 0.0);
    const ExtFacets E = exterior_facets(d, nc, cells);
    std::vector<double> A((size_t)t.n0 * t.n1);
    double xc[12], wc[4];
    for (size_t i = 0; i < E.cell.size(); ++i) {
      const int64_t c = E.cell[i];
      const uint32_t* cell = cells + c * (d + 1);
      gather_coordinates(d, coords, cell, xc);
      gather_vertex_field(d, w, cell, wc);
      t.tabulate(xc, wc, E.local[i], A.data());
      const int32_t* r = dofs0 + c * t.n0;
      const int32_t* cc = dofs1 + c * t.n1;
      for (int a = 0; a < t.n0; ++a)
        for (int b = 0; b < t.n1; ++b)
          if (!csr_add(rowptr, cols, vals, r[a], cc[b], A[a * t.n1 + b])) return -2;
    }
    return 0;
  }
  Tabulator t(*f);
  if (!add_values) std::fill(vals, vals + rowptr[nrows], 0.0);
  std::vector<double> A((size_t)t.n0 * t.n1);
  double xc[12], wc[4], wc2[4];
  for (int64_t c = 0; c < nc; ++c) {
    const uint32_t* cell = cells + c * (d + 1);
    gather_coordinates(d, coords, cell, xc);
    gather_vertex_field(d, w, cell, wc);
    gather_vertex_field(d, w2, cell, wc2);
    t.tabulate(xc, wc, wc2, A.data());
    const int32_t* r = dofs0 + c * t.n0;
    const int32_t* cc = dofs1 + c * t.n1;
    for (int i = 0; i < t.n0; ++i)
      for (int j = 0; j < t.n1; ++j)
        if (!csr_add(rowptr, cols, vals, r[i], cc[j], A[i * t.n1 + j])) return -2;
  }
  return 0;
}

// Vector assembly: Assembler::assemble_cells with EigenVector::add
// (dolfin/la/EigenVector.cpp:160-165).
int orc_assemble_vector(const orc_form* f, int64_t nv, const double* coords, int64_t nc,
                        const uint32_t* cells, const int32_t* dofs0, const double* w,
                        const double* w2, int64_t n, double* b, int add_values) {
  (void)nv;
  const int d = f->tdim;
  if (is_facet_kind(f->kind)) {
    FacetTabulator t(*f);
    if (!add_values) std::fill(b, b + n, 0.0);
    const ExtFacets E = exterior_facets(d, nc, cells);
    std::vector<double> be(t.n0);
    double xc[12], wc[4];
    for (size_t i = 0; i < E.cell.size(); ++i) {
      const int64_t c = E.cell[i];
      const uint32_t* cell = cells + c * (d + 1);
      gather_coordinates(d, coords, cell, xc);
      gather_vertex_field(d, w, cell, wc);
      t.tabulate(xc, wc, E.local[i], be.data());
      const int32_t* r = dofs0 + c * t.n0;
      for (int a = 0; a < t.n0; ++a) b[r[a]] += be[a];
    }
    return 0;
  }
  Tabulator t(*f);
  if (!add_values) std::fill(b, b + n, 0.0);
  std::vector<double> be(t.n0);
  double xc[12], wc[4], wc2[4];
  for (int64_t c = 0; c < nc; ++c) {
    const uint32_t* cell = cells + c * (d + 1);
    gather_coordinates(d, coords, cell, xc);
    gather_vertex_field(d, w, cell, wc);
    gather_vertex_field(d, w2, cell, wc2);
    t.tabulate(xc, wc, wc2, be.data());
    const int32_t* r = dofs0 + c * t.n0;
    for (int i = 0; i < t.n0; ++i) b[r[i]] += be[i];
  }
  return 0;
}

// Functional: assemble(M) for rank-0 forms (Assembler.cpp:186-190 + Scalar::apply).
double orc_assemble_scalar(const orc_form* f, int64_t nv, const double* coords, int64_t nc,
                           const uint32_t* cells, const double* w) {
  (void)nv;
  const int d = f->tdim;
  if (is_facet_kind(f->kind)) {
    FacetTabulator t(*f);
    const ExtFacets E = exterior_facets(d, nc, cells);
    double s = 0.0, a = 0.0, xc[12], wc[4];
    for (size_t i = 0; i < E.cell.size(); ++i) {
      const uint32_t* cell = cells + (int64_t)E.cell[i] * (d + 1);
      gather_coordinates(d, coords, cell, xc);
      gather_vertex_field(d, w, cell, wc);
      t.tabulate(xc, wc, E.local[i], &a);
      s += a;
    }
    return s;
  }
  Tabulator t(*f);
  double s = 0.0, a = 0.0, xc[12], wc[4];
  for (int64_t c = 0; c < nc; ++c) {
    const uint32_t* cell = cells + c * (d + 1);
    gather_coordinates(d, coords, cell, xc);
    gather_vertex_field(d, w, cell, wc);
    t.tabulate(xc, wc, wc, &a);
    s += a;
  }
  return s;
}

// SystemAssembler::cell_wise_assembly (dolfin/fem/SystemAssembler.cpp:303-492)
// for a square a on V x V and L on V, with SystemAssembler::apply_bc
// (:1037-1070, the single-boundary-map branch): per cell, for each local
// column holding a Dirichlet dof: zero the row, subtract column * value from
// the element vector, zero the column, set b_i = value and A_ii = 1.
int orc_assemble_system(const orc_form* a, const orc_form* L, int64_t nv, const double* coords,
                        int64_t nc, const uint32_t* cells, const int32_t* dofs,
                        const double* wa, const double* wL, int64_t nbc, const int32_t* bc_dofs,
                        const double* bc_vals, int64_t n, const int32_t* rowptr,
                        const int32_t* cols, double* vals, double* b) {
  return orc_assemble_system_ds(a, nullptr, L, nullptr, nv, coords, nc, cells, dofs, wa, nullptr,
                                wL, nullptr, nbc, bc_dofs, bc_vals, n, rowptr, cols, vals, b);
}

int orc_assemble_system_ds(const orc_form* a, const orc_form* a_ds, const orc_form* L,
                           const orc_form* L_ds, int64_t nv, const double* coords, int64_t nc,
                           const uint32_t* cells, const int32_t* dofs, const double* wa,
                           const double* wa_ds, const double* wL, const double* wL_ds,
                           int64_t nbc, const int32_t* bc_dofs, const double* bc_vals, int64_t n,
                           const int32_t* rowptr, const int32_t* cols, double* vals, double* b) {
  (void)nv;
  Tabulator ta(*a), tL(*L);
  const int d = a->tdim;
  if (ta.n0 != ta.n1 || ta.n0 != tL.n0) return -1;
  const int k = ta.n0;
  std::unique_ptr<FacetTabulator> tfa, tfL;
  if (a_ds) tfa.reset(new FacetTabulator(*a_ds));
  if (L_ds) tfL.reset(new FacetTabulator(*L_ds));
  if ((tfa && (tfa->n0 != k || tfa->n1 != k)) || (tfL && tfL->n0 != k)) return -1;
  // exterior flag of each (cell, local facet)
  std::vector<uint8_t> ext;
  if (tfa || tfL) {
    ext.assign((size_t)nc * (d + 1), 0);
    const ExtFacets E = exterior_facets(d, nc, cells);
    for (size_t i = 0; i < E.cell.size(); ++i) ext[(size_t)E.cell[i] * (d + 1) + E.local[i]] = 1;
  }
  std::fill(vals, vals + rowptr[n], 0.0);
  std::fill(b, b + n, 0.0);
  std::vector<double> Ae((size_t)k * k), be(k), Af((size_t)k * k), bf(k);
  double xc[12], wc[4], wcL[4], wcf[4];
  auto bc_lookup = [&](int32_t dof, double& v) {
    const int32_t* it = std::lower_bound(bc_dofs, bc_dofs + nbc, dof);
    if (it == bc_dofs + nbc || *it != dof) return false;
    v = bc_vals[it - bc_dofs];
    return true;
  };
  for (int64_t c = 0; c < nc; ++c) {
    const uint32_t* cell = cells + c * (d + 1);
    gather_coordinates(d, coords, cell, xc);
    gather_vertex_field(d, wa, cell, wc);
    gather_vertex_field(d, wL, cell, wcL);
    ta.tabulate(xc, wc, wc, Ae.data());
    tL.tabulate(xc, wcL, wcL, be.data());
    // exterior facets of the cell, in local facet order
    if (!ext.empty())
      for (int fl = 0; fl <= d; ++fl) {
        if (!ext[(size_t)c * (d + 1) + fl]) continue;
        if (tfa) {
          gather_vertex_field(d, wa_ds, cell, wcf);
          tfa->tabulate(xc, wcf, fl, Af.data());
          for (int i = 0; i < k * k; ++i) Ae[i] += Af[i];
        }
        if (tfL) {
          gather_vertex_field(d, wL_ds, cell, wcf);
          tfL->tabulate(xc, wcf, fl, bf.data());
          for (int i = 0; i < k; ++i) be[i] += bf[i];
        }
      }
    const int32_t* cd = dofs + c * k;
    for (int i = 0; i < k; ++i) {
      double g;
      if (!bc_lookup(cd[i], g)) continue;
      for (int j = 0; j < k; ++j) Ae[i * k + j] = 0.0;
      for (int r = 0; r < k; ++r) be[r] -= Ae[r * k + i] * g;
      for (int r = 0; r < k; ++r) Ae[r * k + i] = 0.0;
      be[i] = g;
      Ae[i * k + i] = 1.0;
    }
    for (int i = 0; i < k; ++i) {
      for (int j = 0; j < k; ++j)
        if (!csr_add(rowptr, cols, vals, cd[i], cd[j], Ae[i * k + j])) return -2;
      b[cd[i]] += be[i];
    }
  }
  return 0;
}

int64_t orc_exterior_facets(int tdim, int64_t nc, const uint32_t* cells, uint32_t* facet_cell,
                            int32_t* facet_local) {
  const ExtFacets E = exterior_facets(tdim, nc, cells);
  for (size_t i = 0; i < E.cell.size(); ++i) {
    if (facet_cell) facet_cell[i] = E.cell[i];
    if (facet_local) facet_local[i] = E.local[i];
  }
  return (int64_t)E.cell.size();
}

int64_t orc_boundary_vertices(int gdim, int64_t nv, const double* coords, int32_t* out) {
  int64_t m = 0;
  for (int64_t v = 0; v < nv; ++v) {
    bool on = false;
    for (int r = 0; r < gdim; ++r) {
      const double x = coords[v * gdim + r];
      if (std::fabs(x) < 3e-16 || std::fabs(x - 1.0) < 3e-16) on = true;
    }
    if (on) out[m++] = (int32_t)v;
  }
  return m;
}

// Derivative of the diffusion form with respect to its P1 coefficient
// (the form UFL's derivative(a, kappa, psi) produces: psi * grad(u).grad(v)
// * dx), assembled cell by cell and contracted with the upstream gradient.
int orc_vjp_diffusion(const orc_form* a, int64_t nv, const double* coords, int64_t nc,
                      const uint32_t* cells, const int32_t* dofs, const int32_t* rowptr,
                      const int32_t* cols, const double* gA, const double* f, const double* gb,
                      int load_has_kappa, double* dkappa) {
  const int d = a->tdim;
  std::fill(dkappa, dkappa + nv, 0.0);
  // Tensor of the derivative form: for each local kappa basis psi_m, the
  // element matrix of  psi_m grad(u).grad(v) dx  (a P1 "coefficient" that is
  // the m-th barycentric function), and of  psi_m f v dx  for the load.
  orc_form fa = *a;
  fa.coeff = ORC_COEFF_P1;
  Tabulator ta(fa);
  orc_form fl{};
  fl.kind = ORC_LOAD; fl.tdim = d; fl.gdim = d;
  fl.family0 = a->family0; fl.degree0 = a->degree0; fl.vsize0 = 1;
  fl.coeff = ORC_COEFF_P1_TIMES_P1;
  Tabulator tl(fl);
  const int k = ta.n0;
  std::vector<double> Ae((size_t)k * k), be(k);
  double xc[12], e[4], fc[4];
  for (int64_t c = 0; c < nc; ++c) {
    const uint32_t* cell = cells + c * (d + 1);
    gather_coordinates(d, coords, cell, xc);
    gather_vertex_field(d, f, cell, fc);
    const int32_t* cd = dofs + c * k;
    for (int m = 0; m <= d; ++m) {
      for (int t = 0; t <= d; ++t) e[t] = (t == m) ? 1.0 : 0.0;
      ta.tabulate(xc, e, e, Ae.data());
      double s = 0.0;
      for (int i = 0; i < k; ++i)
        for (int j = 0; j < k; ++j) {
          const int32_t* b0 = cols + rowptr[cd[i]];
          const int32_t* e0 = cols + rowptr[cd[i] + 1];
          const int32_t* it = std::lower_bound(b0, e0, cd[j]);
          if (it == e0 || *it != cd[j]) return -2;
          s += gA[it - cols] * Ae[i * k + j];
        }
      if (load_has_kappa && gb && f) {
        tl.tabulate(xc, e, fc, be.data());
        for (int i = 0; i < k; ++i) s += gb[cd[i]] * be[i];
      }
      dkappa[cell[m]] += s;
    }
  }
  return 0;
}

double orc_quadrature_monomial(int tdim, int degree, int a, int b, int c) {
  Quadrature q = make_quadrature(tdim, degree);
  double s = 0.0;
  for (int p = 0; p < q.size(); ++p) {
    double v = std::pow(q.X[p * tdim], a);
    if (tdim >= 2) v *= std::pow(q.X[p * tdim + 1], b);
    if (tdim >= 3) v *= std::pow(q.X[p * tdim + 2], c);
    s += q.w[p] * v;
  }
  return s;
}

}  // extern "C"
