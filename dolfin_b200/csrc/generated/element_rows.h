// GENERATED by dolfin_b200/codegen/gen_element_rows.py -- do not edit.
//
// Canonical element-matrix rows of the named Lagrange forms, as reference
// tensor (exact rationals) x geometry tensor W.  Row 'v': the row of local
// vertex 0; row 'e': the row of the edge (0,1).  Columns follow the UFC local
// node order of the (relabelled) cell: vertices, then edges in the order of
// TetrahedronCell/TriangleCell::create_entities.
//   grad_grad_*_k1 : out_j = sum_ab W_ab (1/|T|) int dphi_i/dl_a dphi_j/dl_b
//   grad_grad_*_kp1: same with a P1 weight kappa = sum_k kap_k l_k inside
//   load_*_f1      : (1/|T|) int phi_i ;  load_*_fp1: (1/|T|) int f phi_i
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
DB2_HD void grad_grad_p1tri_v_k1(const CT (&W)[1][3], CT (&out)[3]) {
  out[0] = W[0][0];
  out[1] = W[0][1];
  out[2] = W[0][2];
}

template <typename CT>
DB2_HD void grad_grad_p1tri_v_kp1(const CT (&W)[1][3], const CT (&kap)[3], CT (&out)[3]) {
  const CT t0 = ((CT(0.3333333333333333) * kap[0]) + (CT(0.3333333333333333) * kap[1]) + (CT(0.3333333333333333) * kap[2]));
  out[0] = (W[0][0] * t0);
  out[1] = (W[0][1] * t0);
  out[2] = (W[0][2] * t0);
}

template <typename CT>
DB2_HD CT load_p1tri_v_f1() {
  const CT r = CT(0.3333333333333333);
  return r;
}

template <typename CT>
DB2_HD CT load_p1tri_v_fp1(const CT (&f)[3]) {
  const CT r = ((CT(0.16666666666666666) * f[0]) + (CT(0.08333333333333333) * f[1]) + (CT(0.08333333333333333) * f[2]));
  return r;
}

template <typename CT>
DB2_HD void load_p1tri_v_kfp1(const CT (&f)[3], CT (&out)[3]) {
  out[0] = ((CT(0.1) * f[0]) + (CT(0.03333333333333333) * f[1]) + (CT(0.03333333333333333) * f[2]));
  out[1] = ((CT(0.03333333333333333) * f[0]) + (CT(0.03333333333333333) * f[1]) + (CT(0.016666666666666666) * f[2]));
  out[2] = ((CT(0.03333333333333333) * f[0]) + (CT(0.03333333333333333) * f[2]) + (CT(0.016666666666666666) * f[1]));
}

template <typename CT>
DB2_HD void grad_grad_p2tri_v_k1(const CT (&W)[1][3], CT (&out)[6]) {
  out[0] = W[0][0];
  out[1] = (CT(-0.3333333333333333) * W[0][1]);
  out[2] = (CT(-0.3333333333333333) * W[0][2]);
  out[3] = CT(0);
  out[4] = (CT(1.3333333333333333) * W[0][2]);
  out[5] = (CT(1.3333333333333333) * W[0][1]);
}

template <typename CT>
DB2_HD void grad_grad_p2tri_v_kp1(const CT (&W)[1][3], const CT (&kap)[3], CT (&out)[6]) {
  const CT t0 = (CT(3) * kap[0]);
  const CT t1 = (CT(2) * kap[0]);
  const CT t2 = (kap[2] + (CT(2) * kap[1]));
  const CT t3 = (kap[1] + (CT(2) * kap[2]));
  const CT t4 = (CT(-1) * t0);
  const CT t5 = (t3 + t4);
  const CT t6 = (t2 + t4);
  const CT t7 = ((CT(3) * kap[1]) + (CT(3) * kap[2]) + (CT(14) * kap[0]));
  out[0] = (CT(0.2) * W[0][0] * (kap[1] + kap[2] + t0));
  out[1] = (CT(-0.06666666666666667) * W[0][1] * (t1 + t2));
  out[2] = (CT(-0.06666666666666667) * W[0][2] * (t1 + t3));
  out[3] = ((CT(-0.06666666666666667) * W[0][1] * t5) + (CT(-0.06666666666666667) * W[0][2] * t6));
  out[4] = ((CT(-0.06666666666666667) * W[0][0] * t5) + (CT(0.06666666666666667) * W[0][2] * t7));
  out[5] = ((CT(-0.06666666666666667) * W[0][0] * t6) + (CT(0.06666666666666667) * W[0][1] * t7));
}

template <typename CT>
DB2_HD CT load_p2tri_v_f1() {
  const CT r = CT(0);
  return r;
}

template <typename CT>
DB2_HD CT load_p2tri_v_fp1(const CT (&f)[3]) {
  const CT r = ((CT(-0.016666666666666666) * f[1]) + (CT(-0.016666666666666666) * f[2]) + (CT(0.03333333333333333) * f[0]));
  return r;
}

template <typename CT>
DB2_HD void load_p2tri_v_kfp1(const CT (&f)[3], CT (&out)[3]) {
  out[0] = (CT(0.03333333333333333) * f[0]);
  out[1] = ((CT(-0.011111111111111112) * f[1]) + (CT(-0.005555555555555556) * f[2]));
  out[2] = ((CT(-0.011111111111111112) * f[2]) + (CT(-0.005555555555555556) * f[1]));
}

template <typename CT>
DB2_HD void grad_grad_p2tri_e_k1(const CT (&W)[2][3], CT (&out)[6]) {
  out[0] = (CT(1.3333333333333333) * W[1][0]);
  out[1] = (CT(1.3333333333333333) * W[0][1]);
  out[2] = CT(0);
  out[3] = (CT(1.3333333333333333) * (W[0][1] + W[1][1] + W[1][2] + (CT(2) * W[0][2])));
  out[4] = (CT(1.3333333333333333) * (W[0][0] + W[0][2] + W[1][0] + (CT(2) * W[1][2])));
  out[5] = (CT(1.3333333333333333) * (W[0][1] + W[1][0] + (CT(2) * W[0][0]) + (CT(2) * W[1][1])));
}

template <typename CT>
DB2_HD void grad_grad_p2tri_e_kp1(const CT (&W)[2][3], const CT (&kap)[3], CT (&out)[6]) {
  const CT t0 = (CT(3) * kap[0]);
  const CT t1 = (CT(2) * kap[1]);
  const CT t2 = (kap[2] + t1);
  const CT t3 = (CT(3) * kap[1]);
  const CT t4 = (CT(3) * kap[2]);
  const CT t5 = (CT(2) * kap[0]);
  const CT t6 = (CT(-1) * t4);
  const CT t7 = (kap[0] + t1);
  const CT t8 = (kap[1] + t5);
  const CT t9 = ((CT(2) * kap[0]) + (CT(2) * kap[2]) + (CT(2) * t3));
  const CT t10 = (CT(2) * kap[2]);
  const CT t11 = (t10 + t7);
  const CT t12 = (t10 + t8);
  const CT t13 = (t2 + t5);
  const CT t14 = ((CT(2) * kap[1]) + (CT(2) * kap[2]) + (CT(2) * t0));
  out[0] = ((CT(-0.06666666666666667) * W[0][0] * (t2 + (CT(-1) * t0))) + (CT(0.06666666666666667) * W[1][0] * (t3 + t4 + (CT(14) * kap[0]))));
  out[1] = ((CT(-0.06666666666666667) * W[1][1] * (kap[2] + t5 + (CT(-1) * t3))) + (CT(0.06666666666666667) * W[0][1] * (t0 + t4 + (CT(14) * kap[1]))));
  out[2] = ((CT(-0.06666666666666667) * W[0][2] * (t6 + t7)) + (CT(-0.06666666666666667) * W[1][2] * (t6 + t8)));
  out[3] = ((CT(0.26666666666666666) * W[0][1] * t11) + (CT(0.26666666666666666) * W[0][2] * t9) + (CT(0.26666666666666666) * W[1][1] * t12) + (CT(0.26666666666666666) * W[1][2] * t13));
  out[4] = ((CT(0.26666666666666666) * W[0][0] * t11) + (CT(0.26666666666666666) * W[0][2] * t13) + (CT(0.26666666666666666) * W[1][0] * t12) + (CT(0.26666666666666666) * W[1][2] * t14));
  out[5] = ((CT(0.26666666666666666) * W[0][0] * t9) + (CT(0.26666666666666666) * W[0][1] * t13) + (CT(0.26666666666666666) * W[1][0] * t13) + (CT(0.26666666666666666) * W[1][1] * t14));
}

template <typename CT>
DB2_HD CT load_p2tri_e_f1() {
  const CT r = CT(0.3333333333333333);
  return r;
}

template <typename CT>
DB2_HD CT load_p2tri_e_fp1(const CT (&f)[3]) {
  const CT r = ((CT(0.06666666666666667) * f[2]) + (CT(0.13333333333333333) * f[0]) + (CT(0.13333333333333333) * f[1]));
  return r;
}

template <typename CT>
DB2_HD void load_p2tri_e_kfp1(const CT (&f)[3], CT (&out)[3]) {
  out[0] = ((CT(0.06666666666666667) * f[0]) + (CT(0.022222222222222223) * f[2]) + (CT(0.044444444444444446) * f[1]));
  out[1] = ((CT(0.06666666666666667) * f[1]) + (CT(0.022222222222222223) * f[2]) + (CT(0.044444444444444446) * f[0]));
  out[2] = ((CT(0.022222222222222223) * f[0]) + (CT(0.022222222222222223) * f[1]) + (CT(0.022222222222222223) * f[2]));
}

template <typename CT>
DB2_HD void grad_grad_p1tet_v_k1(const CT (&W)[1][4], CT (&out)[4]) {
  out[0] = W[0][0];
  out[1] = W[0][1];
  out[2] = W[0][2];
  out[3] = W[0][3];
}

template <typename CT>
DB2_HD void grad_grad_p1tet_v_kp1(const CT (&W)[1][4], const CT (&kap)[4], CT (&out)[4]) {
  const CT t0 = ((CT(0.25) * kap[0]) + (CT(0.25) * kap[1]) + (CT(0.25) * kap[2]) + (CT(0.25) * kap[3]));
  out[0] = (W[0][0] * t0);
  out[1] = (W[0][1] * t0);
  out[2] = (W[0][2] * t0);
  out[3] = (W[0][3] * t0);
}

template <typename CT>
DB2_HD CT load_p1tet_v_f1() {
  const CT r = CT(0.25);
  return r;
}

template <typename CT>
DB2_HD CT load_p1tet_v_fp1(const CT (&f)[4]) {
  const CT r = ((CT(0.1) * f[0]) + (CT(0.05) * f[1]) + (CT(0.05) * f[2]) + (CT(0.05) * f[3]));
  return r;
}

template <typename CT>
DB2_HD void load_p1tet_v_kfp1(const CT (&f)[4], CT (&out)[4]) {
  out[0] = ((CT(0.05) * f[0]) + (CT(0.016666666666666666) * f[1]) + (CT(0.016666666666666666) * f[2]) + (CT(0.016666666666666666) * f[3]));
  out[1] = ((CT(0.016666666666666666) * f[0]) + (CT(0.016666666666666666) * f[1]) + (CT(0.008333333333333333) * f[2]) + (CT(0.008333333333333333) * f[3]));
  out[2] = ((CT(0.016666666666666666) * f[0]) + (CT(0.016666666666666666) * f[2]) + (CT(0.008333333333333333) * f[1]) + (CT(0.008333333333333333) * f[3]));
  out[3] = ((CT(0.016666666666666666) * f[0]) + (CT(0.016666666666666666) * f[3]) + (CT(0.008333333333333333) * f[1]) + (CT(0.008333333333333333) * f[2]));
}

template <typename CT>
DB2_HD void grad_grad_p2tet_v_k1(const CT (&W)[1][4], CT (&out)[10]) {
  out[0] = (CT(0.6) * W[0][0]);
  out[1] = (CT(-0.2) * W[0][1]);
  out[2] = (CT(-0.2) * W[0][2]);
  out[3] = (CT(-0.2) * W[0][3]);
  out[4] = (CT(-0.2) * (W[0][2] + W[0][3]));
  out[5] = (CT(-0.2) * (W[0][1] + W[0][3]));
  out[6] = (CT(-0.2) * (W[0][1] + W[0][2]));
  out[7] = (CT(0.2) * ((CT(-1) * W[0][0]) + (CT(3) * W[0][3])));
  out[8] = (CT(0.2) * ((CT(-1) * W[0][0]) + (CT(3) * W[0][2])));
  out[9] = (CT(0.2) * ((CT(-1) * W[0][0]) + (CT(3) * W[0][1])));
}

template <typename CT>
DB2_HD void grad_grad_p2tet_v_kp1(const CT (&W)[1][4], const CT (&kap)[4], CT (&out)[10]) {
  const CT t0 = (CT(5) * kap[0]);
  const CT t1 = (kap[3] + t0);
  const CT t2 = (kap[1] + kap[2]);
  const CT t3 = (CT(-1) * kap[0]);
  const CT t4 = (t2 + t3 + (CT(2) * kap[3]));
  const CT t5 = (kap[3] + t3);
  const CT t6 = (kap[1] + t5 + (CT(2) * kap[2]));
  const CT t7 = (kap[2] + t5 + (CT(2) * kap[1]));
  const CT t8 = (kap[3] + t2 + (CT(6) * kap[0]));
  out[0] = (CT(0.016666666666666666) * W[0][0] * ((CT(7) * kap[1]) + (CT(7) * kap[2]) + (CT(7) * kap[3]) + (CT(15) * kap[0])));
  out[1] = (CT(-0.016666666666666666) * W[0][1] * (kap[2] + t1 + (CT(5) * kap[1])));
  out[2] = (CT(-0.016666666666666666) * W[0][2] * (kap[1] + t1 + (CT(5) * kap[2])));
  out[3] = (CT(-0.016666666666666666) * W[0][3] * (t0 + t2 + (CT(5) * kap[3])));
  out[4] = ((CT(-0.06666666666666667) * W[0][2] * t4) + (CT(-0.06666666666666667) * W[0][3] * t6));
  out[5] = ((CT(-0.06666666666666667) * W[0][1] * t4) + (CT(-0.06666666666666667) * W[0][3] * t7));
  out[6] = ((CT(-0.06666666666666667) * W[0][1] * t6) + (CT(-0.06666666666666667) * W[0][2] * t7));
  out[7] = ((CT(-0.06666666666666667) * W[0][0] * t4) + (CT(0.06666666666666667) * W[0][3] * t8));
  out[8] = ((CT(-0.06666666666666667) * W[0][0] * t6) + (CT(0.06666666666666667) * W[0][2] * t8));
  out[9] = ((CT(-0.06666666666666667) * W[0][0] * t7) + (CT(0.06666666666666667) * W[0][1] * t8));
}

template <typename CT>
DB2_HD CT load_p2tet_v_f1() {
  const CT r = CT(-0.05);
  return r;
}

template <typename CT>
DB2_HD CT load_p2tet_v_fp1(const CT (&f)[4]) {
  const CT r = ((CT(-0.016666666666666666) * f[1]) + (CT(-0.016666666666666666) * f[2]) + (CT(-0.016666666666666666) * f[3]));
  return r;
}

template <typename CT>
DB2_HD void load_p2tet_v_kfp1(const CT (&f)[4], CT (&out)[4]) {
  out[0] = ((CT(-0.002380952380952381) * f[1]) + (CT(-0.002380952380952381) * f[2]) + (CT(-0.002380952380952381) * f[3]) + (CT(0.007142857142857143) * f[0]));
  out[1] = ((CT(-0.007142857142857143) * f[1]) + (CT(-0.0035714285714285713) * f[2]) + (CT(-0.0035714285714285713) * f[3]) + (CT(-0.002380952380952381) * f[0]));
  out[2] = ((CT(-0.007142857142857143) * f[2]) + (CT(-0.0035714285714285713) * f[1]) + (CT(-0.0035714285714285713) * f[3]) + (CT(-0.002380952380952381) * f[0]));
  out[3] = ((CT(-0.007142857142857143) * f[3]) + (CT(-0.0035714285714285713) * f[1]) + (CT(-0.0035714285714285713) * f[2]) + (CT(-0.002380952380952381) * f[0]));
}

template <typename CT>
DB2_HD void grad_grad_p2tet_e_k1(const CT (&W)[2][4], CT (&out)[10]) {
  const CT t0 = (W[0][2] + W[1][2]);
  const CT t1 = (W[0][3] + W[1][3]);
  const CT t2 = (W[0][1] + W[1][1]);
  const CT t3 = (W[0][0] + W[1][0]);
  out[0] = (CT(0.2) * ((CT(-1) * W[0][0]) + (CT(3) * W[1][0])));
  out[1] = (CT(0.2) * ((CT(-1) * W[1][1]) + (CT(3) * W[0][1])));
  out[2] = (CT(-0.2) * t0);
  out[3] = (CT(-0.2) * t1);
  out[4] = ((CT(0.8) * t0) + (CT(0.8) * t1));
  out[5] = ((CT(0.8) * W[1][3]) + (CT(0.8) * t2) + (CT(1.6) * W[0][3]));
  out[6] = ((CT(0.8) * W[1][2]) + (CT(0.8) * t2) + (CT(1.6) * W[0][2]));
  out[7] = ((CT(0.8) * W[0][3]) + (CT(0.8) * t3) + (CT(1.6) * W[1][3]));
  out[8] = ((CT(0.8) * W[0][2]) + (CT(0.8) * t3) + (CT(1.6) * W[1][2]));
  out[9] = (CT(0.8) * (W[0][1] + W[1][0] + (CT(2) * W[0][0]) + (CT(2) * W[1][1])));
}

template <typename CT>
DB2_HD void grad_grad_p2tet_e_kp1(const CT (&W)[2][4], const CT (&kap)[4], CT (&out)[10]) {
  const CT t0 = (kap[2] + kap[3]);
  const CT t1 = (kap[1] + t0);
  const CT t2 = (CT(2) * kap[1]);
  const CT t3 = (t0 + t2);
  const CT t4 = (kap[0] + t0);
  const CT t5 = (CT(2) * kap[0]);
  const CT t6 = (kap[3] + (CT(-1) * kap[2]));
  const CT t7 = (kap[0] + t2);
  const CT t8 = (kap[1] + t5);
  const CT t9 = (kap[2] + (CT(-1) * kap[3]));
  const CT t10 = (kap[2] + (CT(2) * kap[3]));
  const CT t11 = (t10 + t7);
  const CT t12 = (kap[3] + (CT(2) * kap[2]));
  const CT t13 = (t12 + t7);
  const CT t14 = (t10 + t8);
  const CT t15 = (t12 + t8);
  const CT t16 = ((CT(2) * t4) + (CT(6) * kap[1]));
  const CT t17 = (t3 + t5);
  const CT t18 = ((CT(2) * t1) + (CT(6) * kap[0]));
  out[0] = ((CT(-0.06666666666666667) * W[0][0] * (t3 + (CT(-1) * kap[0]))) + (CT(0.06666666666666667) * W[1][0] * (t1 + (CT(6) * kap[0]))));
  out[1] = ((CT(-0.06666666666666667) * W[1][1] * (t0 + t5 + (CT(-1) * kap[1]))) + (CT(0.06666666666666667) * W[0][1] * (t4 + (CT(6) * kap[1]))));
  out[2] = ((CT(-0.06666666666666667) * W[0][2] * (t6 + t7)) + (CT(-0.06666666666666667) * W[1][2] * (t6 + t8)));
  out[3] = ((CT(-0.06666666666666667) * W[0][3] * (t7 + t9)) + (CT(-0.06666666666666667) * W[1][3] * (t8 + t9)));
  out[4] = ((CT(0.13333333333333333) * W[0][2] * t11) + (CT(0.13333333333333333) * W[0][3] * t13) + (CT(0.13333333333333333) * W[1][2] * t14) + (CT(0.13333333333333333) * W[1][3] * t15));
  out[5] = ((CT(0.13333333333333333) * W[0][1] * t11) + (CT(0.13333333333333333) * W[0][3] * t16) + (CT(0.13333333333333333) * W[1][1] * t14) + (CT(0.13333333333333333) * W[1][3] * t17));
  out[6] = ((CT(0.13333333333333333) * W[0][1] * t13) + (CT(0.13333333333333333) * W[0][2] * t16) + (CT(0.13333333333333333) * W[1][1] * t15) + (CT(0.13333333333333333) * W[1][2] * t17));
  out[7] = ((CT(0.13333333333333333) * W[0][0] * t11) + (CT(0.13333333333333333) * W[0][3] * t17) + (CT(0.13333333333333333) * W[1][0] * t14) + (CT(0.13333333333333333) * W[1][3] * t18));
  out[8] = ((CT(0.13333333333333333) * W[0][0] * t13) + (CT(0.13333333333333333) * W[0][2] * t17) + (CT(0.13333333333333333) * W[1][0] * t15) + (CT(0.13333333333333333) * W[1][2] * t18));
  out[9] = ((CT(0.13333333333333333) * W[0][0] * t16) + (CT(0.13333333333333333) * W[0][1] * t17) + (CT(0.13333333333333333) * W[1][0] * t17) + (CT(0.13333333333333333) * W[1][1] * t18));
}

template <typename CT>
DB2_HD CT load_p2tet_e_f1() {
  const CT r = CT(0.2);
  return r;
}

template <typename CT>
DB2_HD CT load_p2tet_e_fp1(const CT (&f)[4]) {
  const CT r = ((CT(0.06666666666666667) * f[0]) + (CT(0.06666666666666667) * f[1]) + (CT(0.03333333333333333) * f[2]) + (CT(0.03333333333333333) * f[3]));
  return r;
}

template <typename CT>
DB2_HD void load_p2tet_e_kfp1(const CT (&f)[4], CT (&out)[4]) {
  out[0] = ((CT(0.02857142857142857) * f[0]) + (CT(0.009523809523809525) * f[2]) + (CT(0.009523809523809525) * f[3]) + (CT(0.01904761904761905) * f[1]));
  out[1] = ((CT(0.02857142857142857) * f[1]) + (CT(0.009523809523809525) * f[2]) + (CT(0.009523809523809525) * f[3]) + (CT(0.01904761904761905) * f[0]));
  out[2] = ((CT(0.009523809523809525) * f[0]) + (CT(0.009523809523809525) * f[1]) + (CT(0.009523809523809525) * f[2]) + (CT(0.004761904761904762) * f[3]));
  out[3] = ((CT(0.009523809523809525) * f[0]) + (CT(0.009523809523809525) * f[1]) + (CT(0.009523809523809525) * f[3]) + (CT(0.004761904761904762) * f[2]));
}

}  // namespace gen
}  // namespace db2
