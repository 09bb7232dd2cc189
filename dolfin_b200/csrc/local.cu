// local.cu -- element tensors of selected cells (assemble_local).
//
// LocalAssembler::assemble (dolfin/fem/LocalAssembler.cpp:39-98): the dense
// tensor of one cell in its local dof order (row-major over (test, trial)) --
// the cell integral plus the exterior-facet integrals of the cell's facets
// that lie on the boundary.  Here for a list of cells at once:
//   * cell part: one thread per (cell, test component, local node) relabels
//     the cell so that the node is canonical, evaluates the generated
//     canonical row (the same device code as assembly) and writes it back in
//     local order -- every entry written by exactly one thread;
//   * facet part: one thread per cell adds the rows of its exterior facets.
#include <cuda_runtime.h>

#include "assemble.cuh"
#include "facet_rows.cuh"

namespace db2 {
namespace dev {

// Per local facet fl and facet node t of a cell: the cell-local vertices of
// the relabelled facet (the node canonical) and the cell-local node of each
// relabelled facet node.
struct FacetMaps {
  uint8_t rv[4][6][3];
  uint8_t rn[4][6][6];
};

template <int D, int P, int FORM, bool KP1, int LOADM>
__global__ void __launch_bounds__(256) k_local_cell(const AsmParams p,
                                                    const uint32_t* __restrict__ list,
                                                    int64_t nlist, int64_t nc, int rank,
                                                    double* __restrict__ out) {
  using E = El<D, P>;
  constexpr int K = E::K, NB = D + 1;
  constexpr int BS = FORM == FORM_ELAS ? D : 1;
  constexpr int n = BS * K;
  const int64_t tid = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (tid >= nlist * n) return;
  const int64_t idx = tid / n;
  const int rem = int(tid - idx * n);
  const int c = rem / K, li = rem - c * K;
  const uint32_t cell = __ldg(list + idx);
  if (cell >= nc) return;  // invalid index: its tensor is left unwritten
  uint32_t v[NB], pv[NB];
#pragma unroll
  for (int a = 0; a < NB; ++a) v[a] = __ldg(p.cells + size_t(cell) * NB + a);
  relabel<D>(v, perm_of<D>(li), pv);
  double x[NB][D], kap[NB], fv[NB];
#pragma unroll
  for (int a = 0; a < NB; ++a) {
#pragma unroll
    for (int r = 0; r < D; ++r) x[a][r] = __ldg(p.xw + 4 * size_t(pv[a]) + r);
    kap[a] = KP1 ? __ldg(p.kappa + pv[a]) : 0.0;
    fv[a] = LOADM == LOAD_P1 ? __ldg(p.f + pv[a]) : 0.0;
  }
  Geometry<D> G;
  geometry(x, G);
  const bool vertex = li < NB;
  if (rank == 2) {
    double* row = out + (size_t(idx) * n + c * K + li) * n;
    const uint64_t mc = node_map_of<D, P>(li);
#pragma unroll 1
    for (int e = 0; e < BS; ++e) {
      double o[K];
      element_row<D, P, FORM, KP1, double>(p, G, vertex, c, e, kap, o);
#pragma unroll
      for (int j = 0; j < K; ++j) row[e * K + int((mc >> (4 * j)) & 15u)] = o[j];
    }
  } else {
    out[size_t(idx) * n + c * K + li] = load_row<D, P, LOADM>(p, G, vertex, c, fv, kap);
  }
}

template <int D, int P, bool WP1, bool MATRIX>
__global__ void __launch_bounds__(256) k_local_facets(
    const double* __restrict__ xw, const uint32_t* __restrict__ cells,
    const uint8_t* __restrict__ ext_mask, const FacetMaps F, const uint32_t* __restrict__ list,
    int64_t nlist, int64_t nc, const double* __restrict__ w, double scale, double t0, double t1,
    double t2, int bs, double* __restrict__ out) {
  constexpr int KF = FacetRows<D, P>::KF;
  constexpr int K = El<D, P>::K;
  const int n = bs * K;
  const int64_t idx = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (idx >= nlist) return;
  const uint32_t cell = __ldg(list + idx);
  if (cell >= nc) return;
  const uint32_t mask = __ldg(ext_mask + cell);
  uint32_t cv[D + 1];
#pragma unroll
  for (int a = 0; a <= D; ++a) cv[a] = __ldg(cells + size_t(cell) * (D + 1) + a);
  const double tr[3] = {t0, t1, t2};
  for (int fl = 0; fl <= D; ++fl) {
    if (!(mask >> fl & 1u)) continue;
    for (int t = 0; t < KF; ++t) {
      double x[D][D], wv[D];
#pragma unroll
      for (int a = 0; a < D; ++a) {
        const uint32_t g = cv[F.rv[fl][t][a]];
#pragma unroll
        for (int r = 0; r < D; ++r) x[a][r] = __ldg(xw + 4 * size_t(g) + r);
        wv[a] = WP1 ? __ldg(w + g) : 0.0;
      }
      const bool vertex = t < D;
      const double meas = facet_measure<D>(x);
      const int rowl = F.rn[fl][t][vertex ? 0 : KF - 1];
      if constexpr (MATRIX) {
        double o[KF];
        facet_mass_row<D, P, WP1>(vertex, wv, o);
        double* row = out + (size_t(idx) * n + rowl) * n;
#pragma unroll
        for (int j = 0; j < KF; ++j) row[F.rn[fl][t][j]] += scale * meas * o[j];
      } else {
        const double r = meas * facet_load_row<D, P, WP1>(vertex, wv);
        for (int c = 0; c < bs; ++c) out[size_t(idx) * n + c * K + rowl] += (bs == 1 ? scale : tr[c]) * r;
      }
    }
  }
}

}  // namespace dev

namespace {

// Same canonical facet order and relabelling as the facet assembly plan.
dev::FacetMaps facet_maps(int D, int deg) {
  static const int kCE3[6][2] = {{2, 3}, {1, 3}, {1, 2}, {0, 3}, {0, 2}, {0, 1}};
  static const int kCE2[3][2] = {{1, 2}, {0, 2}, {0, 1}};
  static const int kFE3[3][2] = {{1, 2}, {0, 2}, {0, 1}};
  static const int kFE2[1][2] = {{0, 1}};
  const int (*CE)[2] = D == 3 ? kCE3 : kCE2;
  const int (*FE)[2] = D == 3 ? kFE3 : kFE2;
  const int nce = D == 3 ? 6 : 3, nfe = deg == 2 ? (D == 3 ? 3 : 1) : 0, kf = D + nfe;
  auto cell_edge = [&](int a, int b) {
    for (int e = 0; e < nce; ++e)
      if ((CE[e][0] == a && CE[e][1] == b) || (CE[e][0] == b && CE[e][1] == a)) return e;
    return -1;
  };
  dev::FacetMaps F{};
  for (int fl = 0; fl <= D; ++fl) {
    int av[3], m = 0;
    for (int a = 0; a <= D; ++a)
      if (a != fl) av[m++] = a;
    // cell-local node of facet node s (canonical facet order)
    int fnode[6];
    for (int s = 0; s < D; ++s) fnode[s] = av[s];
    for (int e = 0; e < nfe; ++e) fnode[D + e] = D + 1 + cell_edge(av[FE[e][0]], av[FE[e][1]]);
    auto facet_edge = [&](int p, int q) {
      for (int e = 0; e < nfe; ++e)
        if ((FE[e][0] == p && FE[e][1] == q) || (FE[e][0] == q && FE[e][1] == p)) return e;
      return -1;
    };
    for (int t = 0; t < kf; ++t) {
      int ord[3], mm = 0;
      bool used[3] = {false, false, false};
      auto put = [&](int a) { ord[mm++] = a; used[a] = true; };
      if (t < D) put(t);
      else { put(FE[t - D][0]); put(FE[t - D][1]); }
      for (int a = 0; a < D; ++a)
        if (!used[a]) put(a);
      for (int a = 0; a < D; ++a) F.rv[fl][t][a] = uint8_t(av[ord[a]]);
      for (int j = 0; j < kf; ++j) {
        const int src = j < D ? ord[j] : D + facet_edge(ord[FE[j - D][0]], ord[FE[j - D][1]]);
        F.rn[fl][t][j] = uint8_t(fnode[src]);
      }
    }
  }
  return F;
}

const uint8_t* ext_mask_on_device(Mesh& m) {
  if (!m.d_ext_mask.ptr) {
    m.compute_exterior_facets();
    std::vector<uint8_t> mask(m.nc, 0);
    for (uint32_t e : m.ext_facets) mask[e >> 2] |= uint8_t(1u << (e & 3u));
    m.d_ext_mask.upload(mask.data(), mask.size());
  }
  return m.d_ext_mask.as<uint8_t>();
}

}  // namespace

void launch_local(Space& V, const FormArgs* a, const FormArgs* a_ds, int64_t ncells,
                  const uint32_t* list, double* out, void* stream) {
  Mesh& m = *V.mesh;
  const int D = m.tdim, deg = V.degree, bs = V.vsize;
  const int K = deg == 1 ? D + 1 : (D == 3 ? 10 : 6), n = K * bs;
  if (!a && !a_ds) fail(DB2_ERR_ARGUMENT, "no form");
  auto rank_of = [](int kind) {
    return kind == DB2_FORM_LOAD || kind == DB2_FORM_FACET_LOAD ? 1 : 2;
  };
  const int rank = rank_of(a ? a->f.kind : a_ds->f.kind);
  if (a && a_ds && rank_of(a_ds->f.kind) != rank) fail(DB2_ERR_ARGUMENT, "dx and ds parts of different rank");
  m.ensure_device();
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const size_t total = size_t(ncells) * (rank == 2 ? size_t(n) * n : size_t(n));
  if (ncells <= 0) return;
  if (!a) cudaMemsetAsync(out, 0, total * sizeof(double), s);
  if (a) {
    dev::AsmParams p{};
    p.cells = m.d_cells.as<uint32_t>();
    p.xw = m.d_x.as<double>();
    p.kscale = 1.0;
    bool kp1 = false;
    int loadm = dev::LOAD_NONE;
    int form = dev::FORM_DIFF;
    switch (a->f.kind) {
      case DB2_FORM_DIFFUSION:
        if (bs != 1) fail(DB2_ERR_UNSUPPORTED, "diffusion form on a vector space");
        switch (a->f.coeff) {
          case DB2_COEFF_NONE: break;
          case DB2_COEFF_CONSTANT: p.kscale = a->f.constant[0]; break;
          case DB2_COEFF_P1:
          case DB2_COEFF_P1_SCALED:
            if (!a->w) fail(DB2_ERR_ARGUMENT, "P1 coefficient field missing");
            kp1 = true;
            p.kappa = a->w;
            p.kscale = a->f.coeff == DB2_COEFF_P1 ? 1.0 : a->f.constant[0];
            break;
          default: fail(DB2_ERR_ARGUMENT, "unknown coefficient kind %d", a->f.coeff);
        }
        break;
      case DB2_FORM_ELASTICITY:
        if (D != 3 || bs != 3) fail(DB2_ERR_UNSUPPORTED, "elasticity needs a 3D vector space");
        form = dev::FORM_ELAS;
        p.mu = a->f.mu;
        p.lmbda = a->f.lmbda;
        break;
      case DB2_FORM_LOAD:
        if (a->f.coeff == DB2_COEFF_P1 || a->f.coeff == DB2_COEFF_P1_SCALED) {
          if (bs != 1) fail(DB2_ERR_UNSUPPORTED, "P1 load coefficient on a vector space");
          if (!a->w) fail(DB2_ERR_ARGUMENT, "P1 load field missing");
          loadm = dev::LOAD_P1;
          p.f = a->w;
          p.fc[0] = a->f.coeff == DB2_COEFF_P1 ? 1.0 : a->f.constant[0];
        } else {
          loadm = dev::LOAD_CONST;
          for (int c = 0; c < 3; ++c)
            p.fc[c] = a->f.coeff == DB2_COEFF_NONE ? 1.0 : (bs == 1 ? a->f.constant[0] : a->f.constant[c]);
        }
        if (bs > 1) form = dev::FORM_ELAS;  // vector layout: BS = D test components
        break;
      default: fail(DB2_ERR_UNSUPPORTED, "form kind %d has no cell integral", a->f.kind);
    }
    dev::check_node_maps(D, deg);
    const int64_t nth = ncells * n;
    const unsigned grid = unsigned((nth + 255) / 256);
#define DB2_LC(D_, P_, F_, K_, L_) \
  dev::k_local_cell<D_, P_, F_, K_, L_><<<grid, 256, 0, s>>>(p, list, ncells, m.nc, rank, out)
#define DB2_LC_DP(D_, P_)                                                                    \
  if (D == D_ && deg == P_) {                                                                \
    if (form == dev::FORM_ELAS) {                                                            \
      if constexpr (D_ == 3) {                                                               \
        if (loadm == dev::LOAD_CONST) DB2_LC(3, P_, dev::FORM_ELAS, false, dev::LOAD_CONST); \
        else DB2_LC(3, P_, dev::FORM_ELAS, false, dev::LOAD_NONE);                           \
      } else {                                                                               \
        fail(DB2_ERR_UNSUPPORTED, "vector forms need a 3D mesh");                            \
      }                                                                                      \
    } else if (loadm == dev::LOAD_CONST) {                                                   \
      DB2_LC(D_, P_, dev::FORM_DIFF, false, dev::LOAD_CONST);                                \
    } else if (loadm == dev::LOAD_P1) {                                                      \
      DB2_LC(D_, P_, dev::FORM_DIFF, false, dev::LOAD_P1);                                   \
    } else if (kp1) {                                                                        \
      DB2_LC(D_, P_, dev::FORM_DIFF, true, dev::LOAD_NONE);                                  \
    } else {                                                                                 \
      DB2_LC(D_, P_, dev::FORM_DIFF, false, dev::LOAD_NONE);                                 \
    }                                                                                        \
  }
    DB2_LC_DP(2, 1) DB2_LC_DP(2, 2) DB2_LC_DP(3, 1) DB2_LC_DP(3, 2)
#undef DB2_LC_DP
#undef DB2_LC
    count_launch();
    check_cuda("local cell launch");
  }
  if (a_ds) {
    const FormArgs& f = *a_ds;
    double scale = 1.0, t[3] = {0, 0, 0};
    bool wp1 = false;
    switch (f.f.coeff) {
      case DB2_COEFF_NONE: break;
      case DB2_COEFF_CONSTANT: scale = f.f.constant[0]; break;
      case DB2_COEFF_P1:
      case DB2_COEFF_P1_SCALED:
        if (!f.w) fail(DB2_ERR_ARGUMENT, "P1 facet coefficient field missing");
        wp1 = true;
        scale = f.f.coeff == DB2_COEFF_P1 ? 1.0 : f.f.constant[0];
        break;
      default: fail(DB2_ERR_UNSUPPORTED, "coefficient kind %d for ds forms", f.f.coeff);
    }
    const bool matrix = f.f.kind == DB2_FORM_FACET_MASS;
    if (!matrix && f.f.kind != DB2_FORM_FACET_LOAD) fail(DB2_ERR_ARGUMENT, "not a ds form");
    if (bs != 1) {
      if (matrix || wp1) fail(DB2_ERR_UNSUPPORTED, "vector ds forms take a constant traction");
      for (int c = 0; c < 3; ++c) t[c] = f.f.coeff == DB2_COEFF_NONE ? 1.0 : f.f.constant[c];
    }
    const dev::FacetMaps F = facet_maps(D, deg);
    const uint8_t* mask = ext_mask_on_device(m);
    const unsigned grid = unsigned((ncells + 255) / 256);
    const double* xw = m.d_x.as<double>();
    const uint32_t* cells = m.d_cells.as<uint32_t>();
#define DB2_LF(D_, P_)                                                                           \
  if (D == D_ && deg == P_) {                                                                    \
    if (matrix) {                                                                                \
      if (wp1) dev::k_local_facets<D_, P_, true, true><<<grid, 256, 0, s>>>(                     \
          xw, cells, mask, F, list, ncells, m.nc, f.w, scale, t[0], t[1], t[2], bs, out);              \
      else dev::k_local_facets<D_, P_, false, true><<<grid, 256, 0, s>>>(                        \
          xw, cells, mask, F, list, ncells, m.nc, f.w, scale, t[0], t[1], t[2], bs, out);              \
    } else {                                                                                     \
      if (wp1) dev::k_local_facets<D_, P_, true, false><<<grid, 256, 0, s>>>(                    \
          xw, cells, mask, F, list, ncells, m.nc, f.w, scale, t[0], t[1], t[2], bs, out);              \
      else dev::k_local_facets<D_, P_, false, false><<<grid, 256, 0, s>>>(                       \
          xw, cells, mask, F, list, ncells, m.nc, f.w, scale, t[0], t[1], t[2], bs, out);              \
    }                                                                                            \
  }
    DB2_LF(2, 1) DB2_LF(2, 2) DB2_LF(3, 1) DB2_LF(3, 2)
#undef DB2_LF
    count_launch();
    check_cuda("local facet launch");
  }
}

}  // namespace db2
