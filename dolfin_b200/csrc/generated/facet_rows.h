// GENERATED by dolfin_b200/codegen/gen_facet_rows.py -- do not edit.
//
// Canonical rows of the exterior-facet mass and load tensors, divided by
// the facet measure |F| (see the generator's docstring).
#pragma once
#ifndef DB2_HD
#if defined(__CUDACC__)
#define DB2_HD __host__ __device__ __forceinline__
#else
#define DB2_HD inline
#endif
#endif

namespace db2 {
namespace gen {

template <typename CT>
DB2_HD void facet_mass_p1tri_v_c1(CT (&out)[2]) {
  out[0] = CT(0.3333333333333333);
  out[1] = CT(0.16666666666666666);
}

template <typename CT>
DB2_HD void facet_mass_p1tri_v_cp1(const CT (&w)[2], CT (&out)[2]) {
  out[0] = CT(0.25) * w[0] + CT(0.08333333333333333) * w[1];
  out[1] = CT(0.08333333333333333) * w[0] + CT(0.08333333333333333) * w[1];
}

template <typename CT>
DB2_HD CT facet_load_p1tri_v_c1() {
  return CT(0.5);
}

template <typename CT>
DB2_HD CT facet_load_p1tri_v_cp1(const CT (&w)[2]) {
  return CT(0.3333333333333333) * w[0] + CT(0.16666666666666666) * w[1];
}

template <typename CT>
DB2_HD void facet_mass_p2tri_v_c1(CT (&out)[3]) {
  out[0] = CT(0.13333333333333333);
  out[1] = -CT(0.03333333333333333);
  out[2] = CT(0.06666666666666667);
}

template <typename CT>
DB2_HD void facet_mass_p2tri_v_cp1(const CT (&w)[2], CT (&out)[3]) {
  out[0] = CT(0.016666666666666666) * w[1] + CT(0.11666666666666667) * w[0];
  out[1] = -CT(0.016666666666666666) * w[0] - CT(0.016666666666666666) * w[1];
  out[2] = CT(0.06666666666666667) * w[0];
}

template <typename CT>
DB2_HD CT facet_load_p2tri_v_c1() {
  return CT(0.16666666666666666);
}

template <typename CT>
DB2_HD CT facet_load_p2tri_v_cp1(const CT (&w)[2]) {
  return CT(0.16666666666666666) * w[0];
}

template <typename CT>
DB2_HD void facet_mass_p2tri_e_c1(CT (&out)[3]) {
  out[0] = CT(0.06666666666666667);
  out[1] = CT(0.06666666666666667);
  out[2] = CT(0.5333333333333333);
}

template <typename CT>
DB2_HD void facet_mass_p2tri_e_cp1(const CT (&w)[2], CT (&out)[3]) {
  out[0] = CT(0.06666666666666667) * w[0];
  out[1] = CT(0.06666666666666667) * w[1];
  out[2] = CT(0.26666666666666666) * w[0] + CT(0.26666666666666666) * w[1];
}

template <typename CT>
DB2_HD CT facet_load_p2tri_e_c1() {
  return CT(0.6666666666666666);
}

template <typename CT>
DB2_HD CT facet_load_p2tri_e_cp1(const CT (&w)[2]) {
  return CT(0.3333333333333333) * w[0] + CT(0.3333333333333333) * w[1];
}

template <typename CT>
DB2_HD void facet_mass_p1tet_v_c1(CT (&out)[3]) {
  out[0] = CT(0.16666666666666666);
  out[1] = CT(0.08333333333333333);
  out[2] = CT(0.08333333333333333);
}

template <typename CT>
DB2_HD void facet_mass_p1tet_v_cp1(const CT (&w)[3], CT (&out)[3]) {
  out[0] = CT(0.1) * w[0] + CT(0.03333333333333333) * w[1] + CT(0.03333333333333333) * w[2];
  out[1] = CT(0.03333333333333333) * w[0] + CT(0.03333333333333333) * w[1] + CT(0.016666666666666666) * w[2];
  out[2] = CT(0.03333333333333333) * w[0] + CT(0.03333333333333333) * w[2] + CT(0.016666666666666666) * w[1];
}

template <typename CT>
DB2_HD CT facet_load_p1tet_v_c1() {
  return CT(0.3333333333333333);
}

template <typename CT>
DB2_HD CT facet_load_p1tet_v_cp1(const CT (&w)[3]) {
  return CT(0.16666666666666666) * w[0] + CT(0.08333333333333333) * w[1] + CT(0.08333333333333333) * w[2];
}

template <typename CT>
DB2_HD void facet_mass_p2tet_v_c1(CT (&out)[6]) {
  out[0] = CT(0.03333333333333333);
  out[1] = -CT(0.005555555555555556);
  out[2] = -CT(0.005555555555555556);
  out[3] = -CT(0.022222222222222223);
  out[4] = CT(0);
  out[5] = CT(0);
}

template <typename CT>
DB2_HD void facet_mass_p2tet_v_cp1(const CT (&w)[3], CT (&out)[6]) {
  out[0] = CT(0.023809523809523808) * w[0] + CT(0.004761904761904762) * w[1] + CT(0.004761904761904762) * w[2];
  out[1] = -CT(0.0031746031746031746) * w[0] - CT(0.0031746031746031746) * w[1] + CT(0.0007936507936507937) * w[2];
  out[2] = -CT(0.0031746031746031746) * w[0] - CT(0.0031746031746031746) * w[2] + CT(0.0007936507936507937) * w[1];
  out[3] = -CT(0.009523809523809525) * w[1] - CT(0.009523809523809525) * w[2] - CT(0.0031746031746031746) * w[0];
  out[4] = -CT(0.006349206349206349) * w[2] - CT(0.0031746031746031746) * w[1] + CT(0.009523809523809525) * w[0];
  out[5] = -CT(0.006349206349206349) * w[1] - CT(0.0031746031746031746) * w[2] + CT(0.009523809523809525) * w[0];
}

template <typename CT>
DB2_HD CT facet_load_p2tet_v_c1() {
  return CT(0);
}

template <typename CT>
DB2_HD CT facet_load_p2tet_v_cp1(const CT (&w)[3]) {
  return -CT(0.016666666666666666) * w[1] - CT(0.016666666666666666) * w[2] + CT(0.03333333333333333) * w[0];
}

template <typename CT>
DB2_HD void facet_mass_p2tet_e_c1(CT (&out)[6]) {
  out[0] = CT(0);
  out[1] = CT(0);
  out[2] = -CT(0.022222222222222223);
  out[3] = CT(0.08888888888888889);
  out[4] = CT(0.08888888888888889);
  out[5] = CT(0.17777777777777778);
}

template <typename CT>
DB2_HD void facet_mass_p2tet_e_cp1(const CT (&w)[3], CT (&out)[6]) {
  out[0] = -CT(0.006349206349206349) * w[1] - CT(0.0031746031746031746) * w[2] + CT(0.009523809523809525) * w[0];
  out[1] = -CT(0.006349206349206349) * w[0] - CT(0.0031746031746031746) * w[2] + CT(0.009523809523809525) * w[1];
  out[2] = -CT(0.009523809523809525) * w[0] - CT(0.009523809523809525) * w[1] - CT(0.0031746031746031746) * w[2];
  out[3] = CT(0.0380952380952381) * w[1] + CT(0.025396825396825397) * w[0] + CT(0.025396825396825397) * w[2];
  out[4] = CT(0.0380952380952381) * w[0] + CT(0.025396825396825397) * w[1] + CT(0.025396825396825397) * w[2];
  out[5] = CT(0.0761904761904762) * w[0] + CT(0.0761904761904762) * w[1] + CT(0.025396825396825397) * w[2];
}

template <typename CT>
DB2_HD CT facet_load_p2tet_e_c1() {
  return CT(0.3333333333333333);
}

template <typename CT>
DB2_HD CT facet_load_p2tet_e_cp1(const CT (&w)[3]) {
  return CT(0.06666666666666667) * w[2] + CT(0.13333333333333333) * w[0] + CT(0.13333333333333333) * w[1];
}

}  // namespace gen
}  // namespace db2
