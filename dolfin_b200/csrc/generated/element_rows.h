// GENERATED by dolfin_b200/codegen/gen_element_rows.py -- do not edit.
//
// Canonical element-matrix rows of the named Lagrange forms, as reference
// tensor (exact rationals) x geometry tensor W.  Row 'v': the row of local
// vertex 0; row 'e': the row of the edge (0,1).  Columns follow the UFC local
// node order of the (relabelled) cell: vertices, then edges in the order of
// TetrahedronCell/TriangleCell::create_entities.
//   grad_grad_*_k1 : out_j = sum_ab W_ab (1/|T|) int dphi_i/dl_a dphi_j/dl_b,
//                    called with W * grad_grad_*_scale (integer coefficients remain)
//   grad_grad_*_kp1: same with a P1 weight kappa = sum_k kap_k l_k inside
//   load_*_f1      : (1/|T|) int phi_i ;  load_*_fp1: (1/|T|) int f phi_i
#pragma once
#include <cmath>
#ifndef DB2_HD
#if defined(__CUDACC__)
#define DB2_HD __host__ __device__ __forceinline__
#else
#define DB2_HD inline
#endif
#endif

namespace db2 {
namespace gen {

constexpr double grad_grad_p1tri_v_k1_scale = 1.0;  // 1
template <typename CT>
DB2_HD void grad_grad_p1tri_v_k1(const CT (&W)[1][3], CT (&out)[3]) {
  out[0] = W[0][0];
  out[1] = W[0][1];
  out[2] = W[0][2];
}

constexpr double grad_grad_p1tri_v_kp1_scale = 0.3333333333333333;  // 1/3
template <typename CT>
DB2_HD void grad_grad_p1tri_v_kp1(const CT (&W)[1][3], const CT (&kap)[3], CT (&out)[3]) {
  const CT q0 = (kap[0] + kap[1] + kap[2]);
  out[0] = W[0][0] * q0;
  out[1] = W[0][1] * q0;
  out[2] = W[0][2] * q0;
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

constexpr double grad_grad_p2tri_v_k1_scale = 0.3333333333333333;  // 1/3
template <typename CT>
DB2_HD void grad_grad_p2tri_v_k1(const CT (&W)[1][3], CT (&out)[6]) {
  out[0] = CT(3) * (W[0][0]);
  out[1] = -W[0][1];
  out[2] = -W[0][2];
  out[3] = CT(0);
  out[4] = CT(4) * (W[0][2]);
  out[5] = CT(4) * (W[0][1]);
}

constexpr double grad_grad_p2tri_v_kp1_scale = 0.06666666666666667;  // 1/15
template <typename CT>
DB2_HD void grad_grad_p2tri_v_kp1(const CT (&W)[1][3], const CT (&kap)[3], CT (&out)[6]) {
  const CT t0 = (CT(2) * kap[0]);
  const CT t1 = (kap[2] + (CT(2) * kap[1]));
  const CT t2 = (kap[1] + (CT(2) * kap[2]));
  const CT t3 = (CT(-3) * kap[0]);
  const CT q0 = (kap[1] + kap[2] + (CT(3) * kap[0]));
  const CT q1 = (-t0 - t1);
  const CT q2 = (-t0 - t2);
  const CT q3 = (-t2 - t3);
  const CT q4 = (-t1 - t3);
  const CT q5 = ((CT(3) * kap[1]) + (CT(3) * kap[2]) + (CT(14) * kap[0]));
  out[0] = CT(3) * (W[0][0] * q0);
  out[1] = W[0][1] * q1;
  out[2] = W[0][2] * q2;
  out[3] = fma(W[0][2], q4, W[0][1] * q3);
  out[4] = fma(W[0][2], q5, W[0][0] * q3);
  out[5] = fma(W[0][1], q5, W[0][0] * q4);
}

template <typename CT>
DB2_HD CT load_p2tri_v_f1() {
  const CT r = CT(0);
  return r;
}

template <typename CT>
DB2_HD CT load_p2tri_v_fp1(const CT (&f)[3]) {
  const CT r = (-(CT(0.016666666666666666) * f[1]) - (CT(0.016666666666666666) * f[2]) + (CT(0.03333333333333333) * f[0]));
  return r;
}

template <typename CT>
DB2_HD void load_p2tri_v_kfp1(const CT (&f)[3], CT (&out)[3]) {
  out[0] = (CT(0.03333333333333333) * f[0]);
  out[1] = (-(CT(0.011111111111111112) * f[1]) - (CT(0.005555555555555556) * f[2]));
  out[2] = (-(CT(0.011111111111111112) * f[2]) - (CT(0.005555555555555556) * f[1]));
}

constexpr double grad_grad_p2tri_e_k1_scale = 1.3333333333333333;  // 4/3
template <typename CT>
DB2_HD void grad_grad_p2tri_e_k1(const CT (&W)[2][3], CT (&out)[6]) {
  out[0] = W[1][0];
  out[1] = W[0][1];
  out[2] = CT(0);
  out[3] = ((fma(W[0][2], CT(2), W[0][1]) + W[1][1]) + W[1][2]);
  out[4] = fma(W[1][2], CT(2), ((W[0][0] + W[0][2]) + W[1][0]));
  out[5] = fma(W[1][1], CT(2), ((W[0][0] * CT(2) + W[0][1]) + W[1][0]));
}

constexpr double grad_grad_p2tri_e_kp1_scale = 0.06666666666666667;  // 1/15
template <typename CT>
DB2_HD void grad_grad_p2tri_e_kp1(const CT (&W)[2][3], const CT (&kap)[3], CT (&out)[6]) {
  const CT t0 = (CT(2) * kap[1]);
  const CT t1 = (kap[2] + t0);
  const CT t2 = (CT(3) * kap[1]);
  const CT t3 = (CT(3) * kap[2]);
  const CT t4 = (CT(3) * kap[0]);
  const CT t5 = (CT(2) * kap[0]);
  const CT t6 = (CT(-3) * kap[2]);
  const CT t7 = (kap[0] + t0);
  const CT t8 = (kap[1] + t5);
  const CT t9 = (CT(2) * kap[2]);
  const CT q0 = (-t1 + (CT(3) * kap[0]));
  const CT q1 = (t2 + t3 + (CT(14) * kap[0]));
  const CT q2 = (t3 + t4 + (CT(14) * kap[1]));
  const CT q3 = (-kap[2] - t5 + (CT(3) * kap[1]));
  const CT q4 = (-t6 - t7);
  const CT q5 = (-t6 - t8);
  const CT q6 = (t7 + t9);
  const CT q7 = ((CT(2) * kap[0]) + (CT(2) * kap[2]) + (CT(2) * t2));
  const CT q8 = (t8 + t9);
  const CT q9 = (t1 + t5);
  const CT q10 = ((CT(2) * kap[1]) + (CT(2) * kap[2]) + (CT(2) * t4));
  out[0] = fma(W[1][0], q1, W[0][0] * q0);
  out[1] = fma(W[1][1], q3, W[0][1] * q2);
  out[2] = fma(W[1][2], q5, W[0][2] * q4);
  out[3] = CT(4) * (fma(W[1][2], q9, fma(W[1][1], q8, fma(W[0][2], q7, W[0][1] * q6))));
  out[4] = CT(4) * (fma(W[1][2], q10, fma(W[1][0], q8, fma(W[0][2], q9, W[0][0] * q6))));
  out[5] = CT(4) * (fma(W[1][1], q10, fma(W[1][0], q9, fma(W[0][1], q9, W[0][0] * q7))));
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

constexpr double grad_grad_p1tet_v_k1_scale = 1.0;  // 1
template <typename CT>
DB2_HD void grad_grad_p1tet_v_k1(const CT (&W)[1][4], CT (&out)[4]) {
  out[0] = W[0][0];
  out[1] = W[0][1];
  out[2] = W[0][2];
  out[3] = W[0][3];
}

constexpr double grad_grad_p1tet_v_kp1_scale = 0.25;  // 1/4
template <typename CT>
DB2_HD void grad_grad_p1tet_v_kp1(const CT (&W)[1][4], const CT (&kap)[4], CT (&out)[4]) {
  const CT q0 = (kap[0] + kap[1] + kap[2] + kap[3]);
  out[0] = W[0][0] * q0;
  out[1] = W[0][1] * q0;
  out[2] = W[0][2] * q0;
  out[3] = W[0][3] * q0;
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

constexpr double grad_grad_p2tet_v_k1_scale = 0.2;  // 1/5
template <typename CT>
DB2_HD void grad_grad_p2tet_v_k1(const CT (&W)[1][4], CT (&out)[10]) {
  out[0] = CT(3) * (W[0][0]);
  out[1] = -W[0][1];
  out[2] = -W[0][2];
  out[3] = -W[0][3];
  out[4] = (-W[0][2] - W[0][3]);
  out[5] = (-W[0][1] - W[0][3]);
  out[6] = (-W[0][1] - W[0][2]);
  out[7] = fma(W[0][3], CT(3), -W[0][0]);
  out[8] = fma(W[0][2], CT(3), -W[0][0]);
  out[9] = fma(W[0][1], CT(3), -W[0][0]);
}

constexpr double grad_grad_p2tet_v_kp1_scale = 0.016666666666666666;  // 1/60
template <typename CT>
DB2_HD void grad_grad_p2tet_v_kp1(const CT (&W)[1][4], const CT (&kap)[4], CT (&out)[10]) {
  const CT t0 = (CT(5) * kap[0]);
  const CT t1 = (kap[3] + t0);
  const CT t2 = (kap[1] + kap[2]);
  const CT t3 = (CT(-1) * kap[0]);
  const CT t4 = (kap[3] + t3);
  const CT q0 = ((CT(7) * kap[1]) + (CT(7) * kap[2]) + (CT(7) * kap[3]) + (CT(15) * kap[0]));
  const CT q1 = (-kap[2] - t1 - (CT(5) * kap[1]));
  const CT q2 = (-kap[1] - t1 - (CT(5) * kap[2]));
  const CT q3 = (-t0 - t2 - (CT(5) * kap[3]));
  const CT q4 = (-t2 - t3 - (CT(2) * kap[3]));
  const CT q5 = (-kap[1] - t4 - (CT(2) * kap[2]));
  const CT q6 = (-kap[2] - t4 - (CT(2) * kap[1]));
  const CT q7 = (kap[3] + t2 + (CT(6) * kap[0]));
  out[0] = W[0][0] * q0;
  out[1] = W[0][1] * q1;
  out[2] = W[0][2] * q2;
  out[3] = W[0][3] * q3;
  out[4] = CT(4) * (fma(W[0][3], q5, W[0][2] * q4));
  out[5] = CT(4) * (fma(W[0][3], q6, W[0][1] * q4));
  out[6] = CT(4) * (fma(W[0][2], q6, W[0][1] * q5));
  out[7] = CT(4) * (fma(W[0][3], q7, W[0][0] * q4));
  out[8] = CT(4) * (fma(W[0][2], q7, W[0][0] * q5));
  out[9] = CT(4) * (fma(W[0][1], q7, W[0][0] * q6));
}

template <typename CT>
DB2_HD CT load_p2tet_v_f1() {
  const CT r = CT(-0.05);
  return r;
}

template <typename CT>
DB2_HD CT load_p2tet_v_fp1(const CT (&f)[4]) {
  const CT r = (-(CT(0.016666666666666666) * f[1]) - (CT(0.016666666666666666) * f[2]) - (CT(0.016666666666666666) * f[3]));
  return r;
}

template <typename CT>
DB2_HD void load_p2tet_v_kfp1(const CT (&f)[4], CT (&out)[4]) {
  out[0] = (-(CT(0.002380952380952381) * f[1]) - (CT(0.002380952380952381) * f[2]) - (CT(0.002380952380952381) * f[3]) + (CT(0.007142857142857143) * f[0]));
  out[1] = (-(CT(0.007142857142857143) * f[1]) - (CT(0.0035714285714285713) * f[2]) - (CT(0.0035714285714285713) * f[3]) - (CT(0.002380952380952381) * f[0]));
  out[2] = (-(CT(0.007142857142857143) * f[2]) - (CT(0.0035714285714285713) * f[1]) - (CT(0.0035714285714285713) * f[3]) - (CT(0.002380952380952381) * f[0]));
  out[3] = (-(CT(0.007142857142857143) * f[3]) - (CT(0.0035714285714285713) * f[1]) - (CT(0.0035714285714285713) * f[2]) - (CT(0.002380952380952381) * f[0]));
}

constexpr double grad_grad_p2tet_e_k1_scale = 0.2;  // 1/5
template <typename CT>
DB2_HD void grad_grad_p2tet_e_k1(const CT (&W)[2][4], CT (&out)[10]) {
  out[0] = fma(W[1][0], CT(3), -W[0][0]);
  out[1] = (W[0][1] * CT(3) - W[1][1]);
  out[2] = (-W[0][2] - W[1][2]);
  out[3] = (-W[0][3] - W[1][3]);
  out[4] = CT(4) * ((((W[0][2] + W[0][3]) + W[1][2]) + W[1][3]));
  out[5] = CT(4) * (((fma(W[0][3], CT(2), W[0][1]) + W[1][1]) + W[1][3]));
  out[6] = CT(4) * (((fma(W[0][2], CT(2), W[0][1]) + W[1][1]) + W[1][2]));
  out[7] = CT(4) * (fma(W[1][3], CT(2), ((W[0][0] + W[0][3]) + W[1][0])));
  out[8] = CT(4) * (fma(W[1][2], CT(2), ((W[0][0] + W[0][2]) + W[1][0])));
  out[9] = CT(4) * (fma(W[1][1], CT(2), ((W[0][0] * CT(2) + W[0][1]) + W[1][0])));
}

constexpr double grad_grad_p2tet_e_kp1_scale = 0.06666666666666667;  // 1/15
template <typename CT>
DB2_HD void grad_grad_p2tet_e_kp1(const CT (&W)[2][4], const CT (&kap)[4], CT (&out)[10]) {
  const CT t0 = (CT(2) * kap[1]);
  const CT t1 = (kap[2] + kap[3]);
  const CT t2 = (t0 + t1);
  const CT t3 = (kap[1] + t1);
  const CT t4 = (kap[0] + t1);
  const CT t5 = (CT(2) * kap[0]);
  const CT t6 = (kap[3] - kap[2]);
  const CT t7 = (kap[0] + t0);
  const CT t8 = (kap[1] + t5);
  const CT t9 = (kap[2] - kap[3]);
  const CT t10 = (kap[2] + (CT(2) * kap[3]));
  const CT t11 = (kap[3] + (CT(2) * kap[2]));
  const CT q0 = (kap[0] - t2);
  const CT q1 = (t3 + (CT(6) * kap[0]));
  const CT q2 = (t4 + (CT(6) * kap[1]));
  const CT q3 = (kap[1] - t1 - t5);
  const CT q4 = (-t6 - t7);
  const CT q5 = (-t6 - t8);
  const CT q6 = (-t7 - t9);
  const CT q7 = (-t8 - t9);
  const CT q8 = (t10 + t7);
  const CT q9 = (t11 + t7);
  const CT q10 = (t10 + t8);
  const CT q11 = (t11 + t8);
  const CT q12 = ((CT(2) * t4) + (CT(6) * kap[1]));
  const CT q13 = (t2 + t5);
  const CT q14 = ((CT(2) * t3) + (CT(6) * kap[0]));
  out[0] = fma(W[1][0], q1, W[0][0] * q0);
  out[1] = fma(W[1][1], q3, W[0][1] * q2);
  out[2] = fma(W[1][2], q5, W[0][2] * q4);
  out[3] = fma(W[1][3], q7, W[0][3] * q6);
  out[4] = CT(2) * (fma(W[1][3], q11, fma(W[1][2], q10, fma(W[0][3], q9, W[0][2] * q8))));
  out[5] = CT(2) * (fma(W[1][3], q13, fma(W[1][1], q10, fma(W[0][3], q12, W[0][1] * q8))));
  out[6] = CT(2) * (fma(W[1][2], q13, fma(W[1][1], q11, fma(W[0][2], q12, W[0][1] * q9))));
  out[7] = CT(2) * (fma(W[1][3], q14, fma(W[1][0], q10, fma(W[0][3], q13, W[0][0] * q8))));
  out[8] = CT(2) * (fma(W[1][2], q14, fma(W[1][0], q11, fma(W[0][2], q13, W[0][0] * q9))));
  out[9] = CT(2) * (fma(W[1][1], q14, fma(W[1][0], q13, fma(W[0][1], q13, W[0][0] * q12))));
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
