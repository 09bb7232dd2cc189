// facet_rows.cuh -- device helpers of the exterior-facet kernels: facet
// measure and the generated canonical facet rows (facets.cu, local.cu).
#pragma once

#include <cuda_runtime.h>

#include "generated/facet_rows.h"
#include "internal.h"

namespace db2 {
namespace dev {

// |F|: the length of an edge (2D) or the area of a triangle (3D) given its
// vertices x[a][r].
template <int D>
__device__ __forceinline__ double facet_measure(const double (&x)[D][D]) {
  if constexpr (D == 2) {
    const double dx = x[1][0] - x[0][0], dy = x[1][1] - x[0][1];
    return sqrt(dx * dx + dy * dy);
  } else {
    const double u0 = x[1][0] - x[0][0], u1 = x[1][1] - x[0][1], u2 = x[1][2] - x[0][2];
    const double v0 = x[2][0] - x[0][0], v1 = x[2][1] - x[0][1], v2 = x[2][2] - x[0][2];
    const double c0 = u1 * v2 - u2 * v1, c1 = u2 * v0 - u0 * v2, c2 = u0 * v1 - u1 * v0;
    return 0.5 * sqrt(c0 * c0 + c1 * c1 + c2 * c2);
  }
}

// Generated canonical rows (divided by |F|): KF facet nodes.
template <int D, int P>
struct FacetRows {
  static constexpr int KF = P == 1 ? D : (D == 3 ? 6 : 3);
};

#define DB2_FACET_ROWS_P1(D_, NAME)                                                           \
  template <bool WP1>                                                                        \
  __device__ __forceinline__ double facet_load_row_##NAME(bool, const double (&w)[D_]) {     \
    if constexpr (WP1) return gen::facet_load_##NAME##_v_cp1<double>(w);                     \
    else return gen::facet_load_##NAME##_v_c1<double>();                                     \
  }                                                                                          \
  template <bool WP1>                                                                        \
  __device__ __forceinline__ void facet_mass_row_##NAME(bool, const double (&w)[D_],         \
                                                        double (&o)[FacetRows<D_, 1>::KF]) { \
    if constexpr (WP1) gen::facet_mass_##NAME##_v_cp1<double>(w, o);                         \
    else gen::facet_mass_##NAME##_v_c1<double>(o);                                           \
  }
#define DB2_FACET_ROWS_P2(D_, NAME)                                                           \
  template <bool WP1>                                                                        \
  __device__ __forceinline__ double facet_load_row_##NAME(bool vertex, const double (&w)[D_]) { \
    if constexpr (WP1)                                                                       \
      return vertex ? gen::facet_load_##NAME##_v_cp1<double>(w)                              \
                    : gen::facet_load_##NAME##_e_cp1<double>(w);                             \
    else                                                                                     \
      return vertex ? gen::facet_load_##NAME##_v_c1<double>()                                \
                    : gen::facet_load_##NAME##_e_c1<double>();                               \
  }                                                                                          \
  template <bool WP1>                                                                        \
  __device__ __forceinline__ void facet_mass_row_##NAME(bool vertex, const double (&w)[D_],  \
                                                        double (&o)[FacetRows<D_, 2>::KF]) { \
    if constexpr (WP1) {                                                                     \
      if (vertex) gen::facet_mass_##NAME##_v_cp1<double>(w, o);                              \
      else gen::facet_mass_##NAME##_e_cp1<double>(w, o);                                     \
    } else {                                                                                 \
      if (vertex) gen::facet_mass_##NAME##_v_c1<double>(o);                                  \
      else gen::facet_mass_##NAME##_e_c1<double>(o);                                         \
    }                                                                                        \
  }
DB2_FACET_ROWS_P1(2, p1tri)
DB2_FACET_ROWS_P2(2, p2tri)
DB2_FACET_ROWS_P1(3, p1tet)
DB2_FACET_ROWS_P2(3, p2tet)
#undef DB2_FACET_ROWS_P1
#undef DB2_FACET_ROWS_P2

template <int D, int P, bool WP1>
__device__ __forceinline__ double facet_load_row(bool vertex, const double (&w)[D]) {
  if constexpr (D == 2 && P == 1) return facet_load_row_p1tri<WP1>(vertex, w);
  else if constexpr (D == 2) return facet_load_row_p2tri<WP1>(vertex, w);
  else if constexpr (P == 1) return facet_load_row_p1tet<WP1>(vertex, w);
  else return facet_load_row_p2tet<WP1>(vertex, w);
}

template <int D, int P, bool WP1>
__device__ __forceinline__ void facet_mass_row(bool vertex, const double (&w)[D],
                                               double (&o)[FacetRows<D, P>::KF]) {
  if constexpr (D == 2 && P == 1) facet_mass_row_p1tri<WP1>(vertex, w, o);
  else if constexpr (D == 2) facet_mass_row_p2tri<WP1>(vertex, w, o);
  else if constexpr (P == 1) facet_mass_row_p1tet<WP1>(vertex, w, o);
  else facet_mass_row_p2tet<WP1>(vertex, w, o);
}

}  // namespace dev
}  // namespace db2
