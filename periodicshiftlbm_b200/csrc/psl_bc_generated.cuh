// GENERATED by periodicshiftlbm_b200/csrc/gen_bc.py -- do not edit.
//
// D3Q27 moment-based boundary conditions, one straight-line function per outer
// normal (normal index = (nx+1)*9 + (ny+1)*3 + (nz+1); 13 is the interior).
// Same formulas, evaluated in the same order, as the reference's
// include/boundaryConditions/applyMBBC.h, restoreRho.h, restoreUxUyUz.h,
// restoreRhoUxUyUz.h and the free-slip generator output
// symbolicHelperTools/CppCodeGenerator/results/applyMirror.h.  Every operation is an
// explicit round-to-nearest op (no FMA contraction), and every array index is a
// compile-time constant so the populations stay in registers.
#pragma once

#include "psl_rn.cuh"

namespace psl {
namespace bc {

// ---- outer normal (+1,+0,+0): 9 unknown populations ----
template <typename T>
PSL_HDI void mbbc_n22(T (&f)[27], const T rho, const T ux, const T uy, const T uz) {
  const T smf0 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(f[0], f[1]), f[3]), f[4]), f[5]), f[6]), f[7]), f[9]), f[12]), f[13]), f[14]), f[16]), f[17]), f[18]), f[20]), f[22]), f[23]), f[26]);
  const T smf1 = rn_add(rn_sub(rn_add(rn_sub(rn_sub(rn_add(rn_sub(rn_sub(rn_add(rn_add(rn_add((-f[5]), f[6]), f[12]), f[13]), f[14]), f[16]), f[17]), f[18]), f[20]), f[22]), f[23]), f[26]);
  const T smf2 = rn_add(rn_sub(rn_sub(rn_add(rn_sub(rn_add(rn_add(rn_sub(rn_add(rn_sub(rn_add((-f[3]), f[4]), f[7]), f[9]), f[13]), f[14]), f[17]), f[18]), f[20]), f[22]), f[23]), f[26]);
  const T smf3 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(f[5], f[6]), f[12]), f[13]), f[14]), f[16]), f[17]), f[18]), f[20]), f[22]), f[23]), f[26]);
  const T smf4 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(f[3], f[4]), f[7]), f[9]), f[13]), f[14]), f[17]), f[18]), f[20]), f[22]), f[23]), f[26]);
  const T smf5 = rn_add(rn_add(rn_sub(rn_sub(rn_add(rn_add(rn_sub((-f[13]), f[14]), f[17]), f[18]), f[20]), f[22]), f[23]), f[26]);
  const T smf6 = rn_add(rn_sub(rn_sub(rn_add(rn_sub(rn_add(rn_add((-f[13]), f[14]), f[17]), f[18]), f[20]), f[22]), f[23]), f[26]);
  const T smf7 = rn_add(rn_sub(rn_add(rn_sub(rn_sub(rn_add(rn_sub(f[13], f[14]), f[17]), f[18]), f[20]), f[22]), f[23]), f[26]);
  const T smf8 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(f[13], f[14]), f[17]), f[18]), f[20]), f[22]), f[23]), f[26]);
  const T m0 = rho;
  const T m1 = rn_mul(rho, uy);
  const T m2 = rn_mul(rho, uz);
  const T m3 = rn_add(rn_mul((T(1) / T(3)), rho), rn_mul(rn_mul(rho, uy), uy));
  const T m4 = rn_add(rn_mul((T(1) / T(3)), rho), rn_mul(rn_mul(rho, uz), uz));
  const T m5 = rn_mul(rn_mul(rho, uy), uz);
  const T m6 = rn_add(rn_mul(rn_mul((T(1) / T(3)), rho), uz), rn_mul(rn_mul(rn_mul(rho, uy), uy), uz));
  const T m7 = rn_add(rn_mul(rn_mul((T(1) / T(3)), rho), uy), rn_mul(rn_mul(rn_mul(rho, uy), uz), uz));
  const T m8 = rn_add(rn_add(rn_add(rn_mul((T(1) / T(9)), rho), rn_mul(rn_mul(rn_mul((T(1) / T(3)), rho), uy), uy)), rn_mul(rn_mul(rn_mul((T(1) / T(3)), rho), uz), uz)), rn_mul(rn_mul(rn_mul(rn_mul(rho, uy), uy), uz), uz));
  const T s0 = rn_sub(m0, smf0);
  const T s1 = rn_sub(m1, smf1);
  const T s2 = rn_sub(m2, smf2);
  const T s3 = rn_sub(m3, smf3);
  const T s4 = rn_sub(m4, smf4);
  const T s5 = rn_sub(m5, smf5);
  const T s6 = rn_sub(m6, smf6);
  const T s7 = rn_sub(m7, smf7);
  const T s8 = rn_sub(m8, smf8);
  f[2] = rn_add(rn_sub(rn_sub(s0, s3), s4), s8);
  f[8] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), s2), rn_mul((T(1) / T(2)), s4)), rn_mul((T(-1) / T(2)), s6)), rn_mul((T(-1) / T(2)), s8));
  f[10] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(2)), s2), rn_mul((T(1) / T(2)), s4)), rn_mul((T(1) / T(2)), s6)), rn_mul((T(-1) / T(2)), s8));
  f[11] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(2)), s1), rn_mul((T(1) / T(2)), s3)), rn_mul((T(1) / T(2)), s7)), rn_mul((T(-1) / T(2)), s8));
  f[15] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), s1), rn_mul((T(1) / T(2)), s3)), rn_mul((T(-1) / T(2)), s7)), rn_mul((T(-1) / T(2)), s8));
  f[19] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(4)), s5), rn_mul((T(-1) / T(4)), s6)), rn_mul((T(1) / T(4)), s7)), rn_mul((T(1) / T(4)), s8));
  f[21] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(4)), s5), rn_mul((T(1) / T(4)), s6)), rn_mul((T(-1) / T(4)), s7)), rn_mul((T(1) / T(4)), s8));
  f[24] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(4)), s5), rn_mul((T(1) / T(4)), s6)), rn_mul((T(1) / T(4)), s7)), rn_mul((T(1) / T(4)), s8));
  f[25] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(4)), s5), rn_mul((T(-1) / T(4)), s6)), rn_mul((T(-1) / T(4)), s7)), rn_mul((T(1) / T(4)), s8));
}
template <typename T>
PSL_HDI void restore_rho_u_n22(const T (&f)[27], T& rho, T& ux, T& uy, T& uz) {
  const T q0 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_mul((T(3) / T(2)), f[0]), rn_mul((T(3) / T(2)), f[3])), rn_mul((T(3) / T(2)), f[4])), rn_mul((T(3) / T(2)), f[5])), rn_mul((T(3) / T(2)), f[6])), rn_mul((T(3) / T(2)), f[13])), rn_mul((T(3) / T(2)), f[14])), rn_mul((T(3) / T(2)), f[17])), rn_mul((T(3) / T(2)), f[18]));
  const T q1 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_mul((T(-1) / T(2)), f[0]), rn_mul(T(2), f[1])), rn_mul((T(-1) / T(2)), f[3])), rn_mul((T(-1) / T(2)), f[4])), rn_mul((T(-1) / T(2)), f[5])), rn_mul((T(-1) / T(2)), f[6])), rn_mul(T(2), f[7])), rn_mul(T(2), f[9])), rn_mul(T(2), f[12])), rn_mul((T(-1) / T(2)), f[13])), rn_mul((T(-1) / T(2)), f[14])), rn_mul(T(2), f[16])), rn_mul((T(-1) / T(2)), f[17])), rn_mul((T(-1) / T(2)), f[18])), rn_mul(T(2), f[20])), rn_mul(T(2), f[22])), rn_mul(T(2), f[23])), rn_mul(T(2), f[26]));
  const T q2 = rn_add(rn_add(rn_add(rn_add(rn_sub(rn_add(rn_add(rn_sub(rn_add(rn_add(rn_add((-f[5]), f[6]), rn_mul(T(2), f[12])), f[13]), f[14]), rn_mul(T(-2), f[16])), f[17]), f[18]), rn_mul(T(-2), f[20])), rn_mul(T(2), f[22])), rn_mul(T(-2), f[23])), rn_mul(T(2), f[26]));
  const T q3 = rn_add(rn_add(rn_add(rn_add(rn_sub(rn_add(rn_add(rn_sub(rn_add(rn_add(rn_add((-f[3]), f[4]), rn_mul(T(-2), f[7])), rn_mul(T(2), f[9])), f[13]), f[14]), f[17]), f[18]), rn_mul(T(2), f[20])), rn_mul(T(-2), f[22])), rn_mul(T(-2), f[23])), rn_mul(T(2), f[26]));
  rho = q0;
  ux = rn_div(q1, rho);
  uy = rn_div(q2, rho);
  uz = rn_div(q3, rho);
}
template <typename T>
PSL_HDI void restore_u_n22(const T (&f)[27], const T rho, T& ux, T& uy, T& uz) {
  const T scmf0 = rn_div(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(f[0], rn_mul(T(2), f[1])), f[3]), f[4]), f[5]), f[6]), rn_mul(T(2), f[7])), rn_mul(T(2), f[9])), rn_mul(T(2), f[12])), f[13]), f[14]), rn_mul(T(2), f[16])), f[17]), f[18]), rn_mul(T(2), f[20])), rn_mul(T(2), f[22])), rn_mul(T(2), f[23])), rn_mul(T(2), f[26])), rho);
  const T scmf1 = rn_div(rn_add(rn_add(rn_add(rn_add(rn_sub(rn_add(rn_add(rn_sub(rn_add(rn_add(rn_add((-f[3]), f[4]), rn_mul(T(-2), f[7])), rn_mul(T(2), f[9])), f[13]), f[14]), f[17]), f[18]), rn_mul(T(2), f[20])), rn_mul(T(-2), f[22])), rn_mul(T(-2), f[23])), rn_mul(T(2), f[26])), rho);
  const T scmf2 = rn_div(rn_add(rn_add(rn_add(rn_add(rn_sub(rn_add(rn_add(rn_sub(rn_add(rn_add(rn_add((-f[5]), f[6]), rn_mul(T(2), f[12])), f[13]), f[14]), rn_mul(T(-2), f[16])), f[17]), f[18]), rn_mul(T(-2), f[20])), rn_mul(T(2), f[22])), rn_mul(T(-2), f[23])), rn_mul(T(2), f[26])), rho);
  const T s0 = rn_sub(scmf0, T(1));
  const T s1 = rn_sub(scmf1, T(0));
  const T s2 = rn_sub(scmf2, T(0));
  ux = s0;
  uy = s2;
  uz = s1;
}
template <typename T>
PSL_HDI void restore_rho_n22(const T (&f)[27], T& rho, const T ux, const T uy, const T uz) {
  const T scqu = rn_mul(T(1), ux);
  const T s = rn_add(T(1), scqu);
  const T scmf = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(f[0], rn_mul(T(2), f[1])), f[3]), f[4]), f[5]), f[6]), rn_mul(T(2), f[7])), rn_mul(T(2), f[9])), rn_mul(T(2), f[12])), f[13]), f[14]), rn_mul(T(2), f[16])), f[17]), f[18]), rn_mul(T(2), f[20])), rn_mul(T(2), f[22])), rn_mul(T(2), f[23])), rn_mul(T(2), f[26]));
  rho = rn_div(scmf, s);
}
template <typename T>
PSL_HDI void mirror_n22(T (&f)[27]) {
  f[2] = f[1];
  f[8] = f[9];
  f[10] = f[7];
  f[11] = f[16];
  f[15] = f[12];
  f[19] = f[22];
  f[21] = f[20];
  f[24] = f[26];
  f[25] = f[23];
}

// ---- outer normal (+0,+1,+0): 9 unknown populations ----
template <typename T>
PSL_HDI void mbbc_n16(T (&f)[27], const T rho, const T ux, const T uy, const T uz) {
  const T smf0 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(f[0], f[1]), f[2]), f[3]), f[4]), f[6]), f[7]), f[8]), f[9]), f[10]), f[12]), f[13]), f[15]), f[17]), f[19]), f[22]), f[24]), f[26]);
  const T smf1 = rn_add(rn_sub(rn_add(rn_sub(rn_sub(rn_add(rn_sub(rn_add(rn_sub(rn_add(rn_sub(f[1], f[2]), f[7]), f[8]), f[9]), f[10]), f[12]), f[15]), f[19]), f[22]), f[24]), f[26]);
  const T smf2 = rn_add(rn_add(rn_sub(rn_sub(rn_add(rn_sub(rn_sub(rn_add(rn_add(rn_sub(rn_add((-f[3]), f[4]), f[7]), f[8]), f[9]), f[10]), f[13]), f[17]), f[19]), f[22]), f[24]), f[26]);
  const T smf3 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(f[1], f[2]), f[7]), f[8]), f[9]), f[10]), f[12]), f[15]), f[19]), f[22]), f[24]), f[26]);
  const T smf4 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(f[3], f[4]), f[7]), f[8]), f[9]), f[10]), f[13]), f[17]), f[19]), f[22]), f[24]), f[26]);
  const T smf5 = rn_add(rn_sub(rn_sub(rn_add(rn_add(rn_add(rn_sub((-f[7]), f[8]), f[9]), f[10]), f[19]), f[22]), f[24]), f[26]);
  const T smf6 = rn_add(rn_add(rn_sub(rn_sub(rn_sub(rn_add(rn_add((-f[7]), f[8]), f[9]), f[10]), f[19]), f[22]), f[24]), f[26]);
  const T smf7 = rn_add(rn_sub(rn_add(rn_sub(rn_sub(rn_add(rn_sub(f[7], f[8]), f[9]), f[10]), f[19]), f[22]), f[24]), f[26]);
  const T smf8 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(f[7], f[8]), f[9]), f[10]), f[19]), f[22]), f[24]), f[26]);
  const T m0 = rho;
  const T m1 = rn_mul(rho, ux);
  const T m2 = rn_mul(rho, uz);
  const T m3 = rn_add(rn_mul((T(1) / T(3)), rho), rn_mul(rn_mul(rho, ux), ux));
  const T m4 = rn_add(rn_mul((T(1) / T(3)), rho), rn_mul(rn_mul(rho, uz), uz));
  const T m5 = rn_mul(rn_mul(rho, ux), uz);
  const T m6 = rn_add(rn_mul(rn_mul((T(1) / T(3)), rho), uz), rn_mul(rn_mul(rn_mul(rho, ux), ux), uz));
  const T m7 = rn_add(rn_mul(rn_mul((T(1) / T(3)), rho), ux), rn_mul(rn_mul(rn_mul(rho, ux), uz), uz));
  const T m8 = rn_add(rn_add(rn_add(rn_mul((T(1) / T(9)), rho), rn_mul(rn_mul(rn_mul((T(1) / T(3)), rho), ux), ux)), rn_mul(rn_mul(rn_mul((T(1) / T(3)), rho), uz), uz)), rn_mul(rn_mul(rn_mul(rn_mul(rho, ux), ux), uz), uz));
  const T s0 = rn_sub(m0, smf0);
  const T s1 = rn_sub(m1, smf1);
  const T s2 = rn_sub(m2, smf2);
  const T s3 = rn_sub(m3, smf3);
  const T s4 = rn_sub(m4, smf4);
  const T s5 = rn_sub(m5, smf5);
  const T s6 = rn_sub(m6, smf6);
  const T s7 = rn_sub(m7, smf7);
  const T s8 = rn_sub(m8, smf8);
  f[5] = rn_add(rn_sub(rn_sub(s0, s3), s4), s8);
  f[11] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(2)), s1), rn_mul((T(1) / T(2)), s3)), rn_mul((T(1) / T(2)), s7)), rn_mul((T(-1) / T(2)), s8));
  f[14] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), s2), rn_mul((T(1) / T(2)), s4)), rn_mul((T(-1) / T(2)), s6)), rn_mul((T(-1) / T(2)), s8));
  f[16] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), s1), rn_mul((T(1) / T(2)), s3)), rn_mul((T(-1) / T(2)), s7)), rn_mul((T(-1) / T(2)), s8));
  f[18] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(2)), s2), rn_mul((T(1) / T(2)), s4)), rn_mul((T(1) / T(2)), s6)), rn_mul((T(-1) / T(2)), s8));
  f[20] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(4)), s5), rn_mul((T(1) / T(4)), s6)), rn_mul((T(1) / T(4)), s7)), rn_mul((T(1) / T(4)), s8));
  f[21] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(4)), s5), rn_mul((T(1) / T(4)), s6)), rn_mul((T(-1) / T(4)), s7)), rn_mul((T(1) / T(4)), s8));
  f[23] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(4)), s5), rn_mul((T(-1) / T(4)), s6)), rn_mul((T(1) / T(4)), s7)), rn_mul((T(1) / T(4)), s8));
  f[25] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(4)), s5), rn_mul((T(-1) / T(4)), s6)), rn_mul((T(-1) / T(4)), s7)), rn_mul((T(1) / T(4)), s8));
}
template <typename T>
PSL_HDI void restore_rho_u_n16(const T (&f)[27], T& rho, T& ux, T& uy, T& uz) {
  const T q0 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_mul((T(3) / T(2)), f[0]), rn_mul((T(3) / T(2)), f[1])), rn_mul((T(3) / T(2)), f[2])), rn_mul((T(3) / T(2)), f[3])), rn_mul((T(3) / T(2)), f[4])), rn_mul((T(3) / T(2)), f[7])), rn_mul((T(3) / T(2)), f[8])), rn_mul((T(3) / T(2)), f[9])), rn_mul((T(3) / T(2)), f[10]));
  const T q1 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_sub(rn_add(rn_sub(rn_add(rn_sub(f[1], f[2]), f[7]), f[8]), f[9]), f[10]), rn_mul(T(2), f[12])), rn_mul(T(-2), f[15])), rn_mul(T(-2), f[19])), rn_mul(T(2), f[22])), rn_mul(T(-2), f[24])), rn_mul(T(2), f[26]));
  const T q2 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_mul((T(-1) / T(2)), f[0]), rn_mul((T(-1) / T(2)), f[1])), rn_mul((T(-1) / T(2)), f[2])), rn_mul((T(-1) / T(2)), f[3])), rn_mul((T(-1) / T(2)), f[4])), rn_mul(T(2), f[6])), rn_mul((T(-1) / T(2)), f[7])), rn_mul((T(-1) / T(2)), f[8])), rn_mul((T(-1) / T(2)), f[9])), rn_mul((T(-1) / T(2)), f[10])), rn_mul(T(2), f[12])), rn_mul(T(2), f[13])), rn_mul(T(2), f[15])), rn_mul(T(2), f[17])), rn_mul(T(2), f[19])), rn_mul(T(2), f[22])), rn_mul(T(2), f[24])), rn_mul(T(2), f[26]));
  const T q3 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_sub(rn_add(rn_add(rn_sub(rn_add((-f[3]), f[4]), f[7]), f[8]), f[9]), f[10]), rn_mul(T(-2), f[13])), rn_mul(T(2), f[17])), rn_mul(T(-2), f[19])), rn_mul(T(-2), f[22])), rn_mul(T(2), f[24])), rn_mul(T(2), f[26]));
  rho = q0;
  ux = rn_div(q1, rho);
  uy = rn_div(q2, rho);
  uz = rn_div(q3, rho);
}
template <typename T>
PSL_HDI void restore_u_n16(const T (&f)[27], const T rho, T& ux, T& uy, T& uz) {
  const T scmf0 = rn_div(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(f[0], f[1]), f[2]), f[3]), f[4]), rn_mul(T(2), f[6])), f[7]), f[8]), f[9]), f[10]), rn_mul(T(2), f[12])), rn_mul(T(2), f[13])), rn_mul(T(2), f[15])), rn_mul(T(2), f[17])), rn_mul(T(2), f[19])), rn_mul(T(2), f[22])), rn_mul(T(2), f[24])), rn_mul(T(2), f[26])), rho);
  const T scmf1 = rn_div(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_sub(rn_add(rn_add(rn_sub(rn_add((-f[3]), f[4]), f[7]), f[8]), f[9]), f[10]), rn_mul(T(-2), f[13])), rn_mul(T(2), f[17])), rn_mul(T(-2), f[19])), rn_mul(T(-2), f[22])), rn_mul(T(2), f[24])), rn_mul(T(2), f[26])), rho);
  const T scmf2 = rn_div(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_sub(rn_add(rn_sub(rn_add(rn_sub(f[1], f[2]), f[7]), f[8]), f[9]), f[10]), rn_mul(T(2), f[12])), rn_mul(T(-2), f[15])), rn_mul(T(-2), f[19])), rn_mul(T(2), f[22])), rn_mul(T(-2), f[24])), rn_mul(T(2), f[26])), rho);
  const T s0 = rn_sub(scmf0, T(1));
  const T s1 = rn_sub(scmf1, T(0));
  const T s2 = rn_sub(scmf2, T(0));
  ux = s2;
  uy = s0;
  uz = s1;
}
template <typename T>
PSL_HDI void restore_rho_n16(const T (&f)[27], T& rho, const T ux, const T uy, const T uz) {
  const T scqu = rn_mul(T(1), uy);
  const T s = rn_add(T(1), scqu);
  const T scmf = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(f[0], f[1]), f[2]), f[3]), f[4]), rn_mul(T(2), f[6])), f[7]), f[8]), f[9]), f[10]), rn_mul(T(2), f[12])), rn_mul(T(2), f[13])), rn_mul(T(2), f[15])), rn_mul(T(2), f[17])), rn_mul(T(2), f[19])), rn_mul(T(2), f[22])), rn_mul(T(2), f[24])), rn_mul(T(2), f[26]));
  rho = rn_div(scmf, s);
}
template <typename T>
PSL_HDI void mirror_n16(T (&f)[27]) {
  f[5] = f[6];
  f[11] = f[15];
  f[14] = f[17];
  f[16] = f[12];
  f[18] = f[13];
  f[20] = f[26];
  f[21] = f[24];
  f[23] = f[22];
  f[25] = f[19];
}

// ---- outer normal (+0,+0,+1): 9 unknown populations ----
template <typename T>
PSL_HDI void mbbc_n14(T (&f)[27], const T rho, const T ux, const T uy, const T uz) {
  const T smf0 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(f[0], f[1]), f[2]), f[4]), f[5]), f[6]), f[8]), f[9]), f[11]), f[12]), f[14]), f[15]), f[16]), f[17]), f[20]), f[21]), f[24]), f[26]);
  const T smf1 = rn_add(rn_sub(rn_sub(rn_add(rn_add(rn_sub(rn_add(rn_sub(rn_add(rn_sub(rn_sub(f[1], f[2]), f[8]), f[9]), f[11]), f[12]), f[15]), f[16]), f[20]), f[21]), f[24]), f[26]);
  const T smf2 = rn_add(rn_add(rn_sub(rn_sub(rn_add(rn_sub(rn_add(rn_sub(rn_add(rn_sub(rn_add((-f[5]), f[6]), f[11]), f[12]), f[14]), f[15]), f[16]), f[17]), f[20]), f[21]), f[24]), f[26]);
  const T smf3 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(f[1], f[2]), f[8]), f[9]), f[11]), f[12]), f[15]), f[16]), f[20]), f[21]), f[24]), f[26]);
  const T smf4 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(f[5], f[6]), f[11]), f[12]), f[14]), f[15]), f[16]), f[17]), f[20]), f[21]), f[24]), f[26]);
  const T smf5 = rn_add(rn_sub(rn_add(rn_sub(rn_sub(rn_sub(rn_add(f[11], f[12]), f[15]), f[16]), f[20]), f[21]), f[24]), f[26]);
  const T smf6 = rn_add(rn_add(rn_sub(rn_sub(rn_sub(rn_add(rn_add((-f[11]), f[12]), f[15]), f[16]), f[20]), f[21]), f[24]), f[26]);
  const T smf7 = rn_add(rn_sub(rn_sub(rn_add(rn_add(rn_sub(rn_add((-f[11]), f[12]), f[15]), f[16]), f[20]), f[21]), f[24]), f[26]);
  const T smf8 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(f[11], f[12]), f[15]), f[16]), f[20]), f[21]), f[24]), f[26]);
  const T m0 = rho;
  const T m1 = rn_mul(rho, ux);
  const T m2 = rn_mul(rho, uy);
  const T m3 = rn_add(rn_mul((T(1) / T(3)), rho), rn_mul(rn_mul(rho, ux), ux));
  const T m4 = rn_add(rn_mul((T(1) / T(3)), rho), rn_mul(rn_mul(rho, uy), uy));
  const T m5 = rn_mul(rn_mul(rho, ux), uy);
  const T m6 = rn_add(rn_mul(rn_mul((T(1) / T(3)), rho), uy), rn_mul(rn_mul(rn_mul(rho, ux), ux), uy));
  const T m7 = rn_add(rn_mul(rn_mul((T(1) / T(3)), rho), ux), rn_mul(rn_mul(rn_mul(rho, ux), uy), uy));
  const T m8 = rn_add(rn_add(rn_add(rn_mul((T(1) / T(9)), rho), rn_mul(rn_mul(rn_mul((T(1) / T(3)), rho), ux), ux)), rn_mul(rn_mul(rn_mul((T(1) / T(3)), rho), uy), uy)), rn_mul(rn_mul(rn_mul(rn_mul(rho, ux), ux), uy), uy));
  const T s0 = rn_sub(m0, smf0);
  const T s1 = rn_sub(m1, smf1);
  const T s2 = rn_sub(m2, smf2);
  const T s3 = rn_sub(m3, smf3);
  const T s4 = rn_sub(m4, smf4);
  const T s5 = rn_sub(m5, smf5);
  const T s6 = rn_sub(m6, smf6);
  const T s7 = rn_sub(m7, smf7);
  const T s8 = rn_sub(m8, smf8);
  f[3] = rn_add(rn_sub(rn_sub(s0, s3), s4), s8);
  f[7] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), s1), rn_mul((T(1) / T(2)), s3)), rn_mul((T(-1) / T(2)), s7)), rn_mul((T(-1) / T(2)), s8));
  f[10] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(2)), s1), rn_mul((T(1) / T(2)), s3)), rn_mul((T(1) / T(2)), s7)), rn_mul((T(-1) / T(2)), s8));
  f[13] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), s2), rn_mul((T(1) / T(2)), s4)), rn_mul((T(-1) / T(2)), s6)), rn_mul((T(-1) / T(2)), s8));
  f[18] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(2)), s2), rn_mul((T(1) / T(2)), s4)), rn_mul((T(1) / T(2)), s6)), rn_mul((T(-1) / T(2)), s8));
  f[19] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(4)), s5), rn_mul((T(1) / T(4)), s6)), rn_mul((T(-1) / T(4)), s7)), rn_mul((T(1) / T(4)), s8));
  f[22] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(4)), s5), rn_mul((T(1) / T(4)), s6)), rn_mul((T(1) / T(4)), s7)), rn_mul((T(1) / T(4)), s8));
  f[23] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(4)), s5), rn_mul((T(-1) / T(4)), s6)), rn_mul((T(1) / T(4)), s7)), rn_mul((T(1) / T(4)), s8));
  f[25] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(4)), s5), rn_mul((T(-1) / T(4)), s6)), rn_mul((T(-1) / T(4)), s7)), rn_mul((T(1) / T(4)), s8));
}
template <typename T>
PSL_HDI void restore_rho_u_n14(const T (&f)[27], T& rho, T& ux, T& uy, T& uz) {
  const T q0 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_mul((T(3) / T(2)), f[0]), rn_mul((T(3) / T(2)), f[1])), rn_mul((T(3) / T(2)), f[2])), rn_mul((T(3) / T(2)), f[5])), rn_mul((T(3) / T(2)), f[6])), rn_mul((T(3) / T(2)), f[11])), rn_mul((T(3) / T(2)), f[12])), rn_mul((T(3) / T(2)), f[15])), rn_mul((T(3) / T(2)), f[16]));
  const T q1 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_sub(rn_add(rn_sub(rn_add(rn_add(rn_sub(f[1], f[2]), rn_mul(T(-2), f[8])), rn_mul(T(2), f[9])), f[11]), f[12]), f[15]), f[16]), rn_mul(T(2), f[20])), rn_mul(T(-2), f[21])), rn_mul(T(-2), f[24])), rn_mul(T(2), f[26]));
  const T q2 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_sub(rn_add(rn_add(rn_add(rn_sub(rn_add((-f[5]), f[6]), f[11]), f[12]), rn_mul(T(-2), f[14])), f[15]), f[16]), rn_mul(T(2), f[17])), rn_mul(T(-2), f[20])), rn_mul(T(-2), f[21])), rn_mul(T(2), f[24])), rn_mul(T(2), f[26]));
  const T q3 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_mul((T(-1) / T(2)), f[0]), rn_mul((T(-1) / T(2)), f[1])), rn_mul((T(-1) / T(2)), f[2])), rn_mul(T(2), f[4])), rn_mul((T(-1) / T(2)), f[5])), rn_mul((T(-1) / T(2)), f[6])), rn_mul(T(2), f[8])), rn_mul(T(2), f[9])), rn_mul((T(-1) / T(2)), f[11])), rn_mul((T(-1) / T(2)), f[12])), rn_mul(T(2), f[14])), rn_mul((T(-1) / T(2)), f[15])), rn_mul((T(-1) / T(2)), f[16])), rn_mul(T(2), f[17])), rn_mul(T(2), f[20])), rn_mul(T(2), f[21])), rn_mul(T(2), f[24])), rn_mul(T(2), f[26]));
  rho = q0;
  ux = rn_div(q1, rho);
  uy = rn_div(q2, rho);
  uz = rn_div(q3, rho);
}
template <typename T>
PSL_HDI void restore_u_n14(const T (&f)[27], const T rho, T& ux, T& uy, T& uz) {
  const T scmf0 = rn_div(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(f[0], f[1]), f[2]), rn_mul(T(2), f[4])), f[5]), f[6]), rn_mul(T(2), f[8])), rn_mul(T(2), f[9])), f[11]), f[12]), rn_mul(T(2), f[14])), f[15]), f[16]), rn_mul(T(2), f[17])), rn_mul(T(2), f[20])), rn_mul(T(2), f[21])), rn_mul(T(2), f[24])), rn_mul(T(2), f[26])), rho);
  const T scmf1 = rn_div(rn_add(rn_add(rn_add(rn_add(rn_add(rn_sub(rn_add(rn_add(rn_add(rn_sub(rn_add((-f[5]), f[6]), f[11]), f[12]), rn_mul(T(-2), f[14])), f[15]), f[16]), rn_mul(T(2), f[17])), rn_mul(T(-2), f[20])), rn_mul(T(-2), f[21])), rn_mul(T(2), f[24])), rn_mul(T(2), f[26])), rho);
  const T scmf2 = rn_div(rn_add(rn_add(rn_add(rn_add(rn_add(rn_sub(rn_add(rn_sub(rn_add(rn_add(rn_sub(f[1], f[2]), rn_mul(T(-2), f[8])), rn_mul(T(2), f[9])), f[11]), f[12]), f[15]), f[16]), rn_mul(T(2), f[20])), rn_mul(T(-2), f[21])), rn_mul(T(-2), f[24])), rn_mul(T(2), f[26])), rho);
  const T s0 = rn_sub(scmf0, T(1));
  const T s1 = rn_sub(scmf1, T(0));
  const T s2 = rn_sub(scmf2, T(0));
  ux = s2;
  uy = s1;
  uz = s0;
}
template <typename T>
PSL_HDI void restore_rho_n14(const T (&f)[27], T& rho, const T ux, const T uy, const T uz) {
  const T scqu = rn_mul(T(1), uz);
  const T s = rn_add(T(1), scqu);
  const T scmf = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(f[0], f[1]), f[2]), rn_mul(T(2), f[4])), f[5]), f[6]), rn_mul(T(2), f[8])), rn_mul(T(2), f[9])), f[11]), f[12]), rn_mul(T(2), f[14])), f[15]), f[16]), rn_mul(T(2), f[17])), rn_mul(T(2), f[20])), rn_mul(T(2), f[21])), rn_mul(T(2), f[24])), rn_mul(T(2), f[26]));
  rho = rn_div(scmf, s);
}
template <typename T>
PSL_HDI void mirror_n14(T (&f)[27]) {
  f[3] = f[4];
  f[7] = f[9];
  f[10] = f[8];
  f[13] = f[17];
  f[18] = f[14];
  f[19] = f[24];
  f[22] = f[26];
  f[23] = f[20];
  f[25] = f[21];
}

// ---- outer normal (-1,+0,+0): 9 unknown populations ----
template <typename T>
PSL_HDI void mbbc_n4(T (&f)[27], const T rho, const T ux, const T uy, const T uz) {
  const T smf0 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(f[0], f[2]), f[3]), f[4]), f[5]), f[6]), f[8]), f[10]), f[11]), f[13]), f[14]), f[15]), f[17]), f[18]), f[19]), f[21]), f[24]), f[25]);
  const T smf1 = rn_sub(rn_add(rn_sub(rn_add(rn_sub(rn_add(rn_add(rn_sub(rn_add(rn_sub(rn_add((-f[5]), f[6]), f[11]), f[13]), f[14]), f[15]), f[17]), f[18]), f[19]), f[21]), f[24]), f[25]);
  const T smf2 = rn_sub(rn_add(rn_add(rn_sub(rn_sub(rn_add(rn_add(rn_sub(rn_sub(rn_add(rn_add((-f[3]), f[4]), f[8]), f[10]), f[13]), f[14]), f[17]), f[18]), f[19]), f[21]), f[24]), f[25]);
  const T smf3 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(f[5], f[6]), f[11]), f[13]), f[14]), f[15]), f[17]), f[18]), f[19]), f[21]), f[24]), f[25]);
  const T smf4 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(f[3], f[4]), f[8]), f[10]), f[13]), f[14]), f[17]), f[18]), f[19]), f[21]), f[24]), f[25]);
  const T smf5 = rn_add(rn_add(rn_sub(rn_sub(rn_add(rn_add(rn_sub((-f[13]), f[14]), f[17]), f[18]), f[19]), f[21]), f[24]), f[25]);
  const T smf6 = rn_sub(rn_add(rn_add(rn_sub(rn_sub(rn_add(rn_add((-f[13]), f[14]), f[17]), f[18]), f[19]), f[21]), f[24]), f[25]);
  const T smf7 = rn_sub(rn_add(rn_sub(rn_add(rn_sub(rn_add(rn_sub(f[13], f[14]), f[17]), f[18]), f[19]), f[21]), f[24]), f[25]);
  const T smf8 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(f[13], f[14]), f[17]), f[18]), f[19]), f[21]), f[24]), f[25]);
  const T m0 = rho;
  const T m1 = rn_mul(rho, uy);
  const T m2 = rn_mul(rho, uz);
  const T m3 = rn_add(rn_mul((T(1) / T(3)), rho), rn_mul(rn_mul(rho, uy), uy));
  const T m4 = rn_add(rn_mul((T(1) / T(3)), rho), rn_mul(rn_mul(rho, uz), uz));
  const T m5 = rn_mul(rn_mul(rho, uy), uz);
  const T m6 = rn_add(rn_mul(rn_mul((T(1) / T(3)), rho), uz), rn_mul(rn_mul(rn_mul(rho, uy), uy), uz));
  const T m7 = rn_add(rn_mul(rn_mul((T(1) / T(3)), rho), uy), rn_mul(rn_mul(rn_mul(rho, uy), uz), uz));
  const T m8 = rn_add(rn_add(rn_add(rn_mul((T(1) / T(9)), rho), rn_mul(rn_mul(rn_mul((T(1) / T(3)), rho), uy), uy)), rn_mul(rn_mul(rn_mul((T(1) / T(3)), rho), uz), uz)), rn_mul(rn_mul(rn_mul(rn_mul(rho, uy), uy), uz), uz));
  const T s0 = rn_sub(m0, smf0);
  const T s1 = rn_sub(m1, smf1);
  const T s2 = rn_sub(m2, smf2);
  const T s3 = rn_sub(m3, smf3);
  const T s4 = rn_sub(m4, smf4);
  const T s5 = rn_sub(m5, smf5);
  const T s6 = rn_sub(m6, smf6);
  const T s7 = rn_sub(m7, smf7);
  const T s8 = rn_sub(m8, smf8);
  f[1] = rn_add(rn_sub(rn_sub(s0, s3), s4), s8);
  f[7] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(2)), s2), rn_mul((T(1) / T(2)), s4)), rn_mul((T(1) / T(2)), s6)), rn_mul((T(-1) / T(2)), s8));
  f[9] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), s2), rn_mul((T(1) / T(2)), s4)), rn_mul((T(-1) / T(2)), s6)), rn_mul((T(-1) / T(2)), s8));
  f[12] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), s1), rn_mul((T(1) / T(2)), s3)), rn_mul((T(-1) / T(2)), s7)), rn_mul((T(-1) / T(2)), s8));
  f[16] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(2)), s1), rn_mul((T(1) / T(2)), s3)), rn_mul((T(1) / T(2)), s7)), rn_mul((T(-1) / T(2)), s8));
  f[20] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(4)), s5), rn_mul((T(1) / T(4)), s6)), rn_mul((T(-1) / T(4)), s7)), rn_mul((T(1) / T(4)), s8));
  f[22] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(4)), s5), rn_mul((T(-1) / T(4)), s6)), rn_mul((T(1) / T(4)), s7)), rn_mul((T(1) / T(4)), s8));
  f[23] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(4)), s5), rn_mul((T(-1) / T(4)), s6)), rn_mul((T(-1) / T(4)), s7)), rn_mul((T(1) / T(4)), s8));
  f[26] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(4)), s5), rn_mul((T(1) / T(4)), s6)), rn_mul((T(1) / T(4)), s7)), rn_mul((T(1) / T(4)), s8));
}
template <typename T>
PSL_HDI void restore_rho_u_n4(const T (&f)[27], T& rho, T& ux, T& uy, T& uz) {
  const T q0 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_mul((T(3) / T(2)), f[0]), rn_mul((T(3) / T(2)), f[3])), rn_mul((T(3) / T(2)), f[4])), rn_mul((T(3) / T(2)), f[5])), rn_mul((T(3) / T(2)), f[6])), rn_mul((T(3) / T(2)), f[13])), rn_mul((T(3) / T(2)), f[14])), rn_mul((T(3) / T(2)), f[17])), rn_mul((T(3) / T(2)), f[18]));
  const T q1 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), f[0]), rn_mul(T(-2), f[2])), rn_mul((T(1) / T(2)), f[3])), rn_mul((T(1) / T(2)), f[4])), rn_mul((T(1) / T(2)), f[5])), rn_mul((T(1) / T(2)), f[6])), rn_mul(T(-2), f[8])), rn_mul(T(-2), f[10])), rn_mul(T(-2), f[11])), rn_mul((T(1) / T(2)), f[13])), rn_mul((T(1) / T(2)), f[14])), rn_mul(T(-2), f[15])), rn_mul((T(1) / T(2)), f[17])), rn_mul((T(1) / T(2)), f[18])), rn_mul(T(-2), f[19])), rn_mul(T(-2), f[21])), rn_mul(T(-2), f[24])), rn_mul(T(-2), f[25]));
  const T q2 = rn_add(rn_add(rn_add(rn_add(rn_sub(rn_add(rn_add(rn_sub(rn_add(rn_add(rn_add((-f[5]), f[6]), rn_mul(T(-2), f[11])), f[13]), f[14]), rn_mul(T(2), f[15])), f[17]), f[18]), rn_mul(T(2), f[19])), rn_mul(T(-2), f[21])), rn_mul(T(2), f[24])), rn_mul(T(-2), f[25]));
  const T q3 = rn_add(rn_add(rn_add(rn_add(rn_sub(rn_add(rn_add(rn_sub(rn_add(rn_add(rn_add((-f[3]), f[4]), rn_mul(T(2), f[8])), rn_mul(T(-2), f[10])), f[13]), f[14]), f[17]), f[18]), rn_mul(T(-2), f[19])), rn_mul(T(2), f[21])), rn_mul(T(2), f[24])), rn_mul(T(-2), f[25]));
  rho = q0;
  ux = rn_div(q1, rho);
  uy = rn_div(q2, rho);
  uz = rn_div(q3, rho);
}
template <typename T>
PSL_HDI void restore_u_n4(const T (&f)[27], const T rho, T& ux, T& uy, T& uz) {
  const T scmf0 = rn_div(rn_add(rn_add(rn_add(rn_add(rn_sub(rn_sub(rn_add(rn_sub(rn_sub(rn_add(rn_add(rn_add(rn_sub(rn_sub(rn_sub(rn_sub(rn_add((-f[0]), rn_mul(T(-2), f[2])), f[3]), f[4]), f[5]), f[6]), rn_mul(T(-2), f[8])), rn_mul(T(-2), f[10])), rn_mul(T(-2), f[11])), f[13]), f[14]), rn_mul(T(-2), f[15])), f[17]), f[18]), rn_mul(T(-2), f[19])), rn_mul(T(-2), f[21])), rn_mul(T(-2), f[24])), rn_mul(T(-2), f[25])), rho);
  const T scmf1 = rn_div(rn_add(rn_add(rn_add(rn_add(rn_add(rn_sub(rn_sub(rn_add(rn_add(rn_add(rn_sub(f[3], f[4]), rn_mul(T(-2), f[8])), rn_mul(T(2), f[10])), f[13]), f[14]), f[17]), f[18]), rn_mul(T(2), f[19])), rn_mul(T(-2), f[21])), rn_mul(T(-2), f[24])), rn_mul(T(2), f[25])), rho);
  const T scmf2 = rn_div(rn_add(rn_add(rn_add(rn_add(rn_add(rn_sub(rn_add(rn_add(rn_sub(rn_add(rn_sub(f[5], f[6]), rn_mul(T(2), f[11])), f[13]), f[14]), rn_mul(T(-2), f[15])), f[17]), f[18]), rn_mul(T(-2), f[19])), rn_mul(T(2), f[21])), rn_mul(T(-2), f[24])), rn_mul(T(2), f[25])), rho);
  const T s0 = rn_sub(scmf0, T(-1));
  const T s1 = rn_sub(scmf1, T(0));
  const T s2 = rn_sub(scmf2, T(0));
  ux = s0;
  uy = (-s2);
  uz = (-s1);
}
template <typename T>
PSL_HDI void restore_rho_n4(const T (&f)[27], T& rho, const T ux, const T uy, const T uz) {
  const T scqu = rn_mul(T(1), ux);
  const T s = rn_add(T(-1), scqu);
  const T scmf = rn_add(rn_add(rn_add(rn_add(rn_sub(rn_sub(rn_add(rn_sub(rn_sub(rn_add(rn_add(rn_add(rn_sub(rn_sub(rn_sub(rn_sub(rn_add((-f[0]), rn_mul(T(-2), f[2])), f[3]), f[4]), f[5]), f[6]), rn_mul(T(-2), f[8])), rn_mul(T(-2), f[10])), rn_mul(T(-2), f[11])), f[13]), f[14]), rn_mul(T(-2), f[15])), f[17]), f[18]), rn_mul(T(-2), f[19])), rn_mul(T(-2), f[21])), rn_mul(T(-2), f[24])), rn_mul(T(-2), f[25]));
  rho = rn_div(scmf, s);
}
template <typename T>
PSL_HDI void mirror_n4(T (&f)[27]) {
  f[1] = f[2];
  f[7] = f[10];
  f[9] = f[8];
  f[12] = f[15];
  f[16] = f[11];
  f[20] = f[21];
  f[22] = f[19];
  f[23] = f[25];
  f[26] = f[24];
}

// ---- outer normal (+0,-1,+0): 9 unknown populations ----
template <typename T>
PSL_HDI void mbbc_n10(T (&f)[27], const T rho, const T ux, const T uy, const T uz) {
  const T smf0 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(f[0], f[1]), f[2]), f[3]), f[4]), f[5]), f[7]), f[8]), f[9]), f[10]), f[11]), f[14]), f[16]), f[18]), f[20]), f[21]), f[23]), f[25]);
  const T smf1 = rn_sub(rn_add(rn_sub(rn_add(rn_add(rn_sub(rn_sub(rn_add(rn_sub(rn_add(rn_sub(f[1], f[2]), f[7]), f[8]), f[9]), f[10]), f[11]), f[16]), f[20]), f[21]), f[23]), f[25]);
  const T smf2 = rn_sub(rn_sub(rn_add(rn_add(rn_sub(rn_add(rn_sub(rn_add(rn_add(rn_sub(rn_add((-f[3]), f[4]), f[7]), f[8]), f[9]), f[10]), f[14]), f[18]), f[20]), f[21]), f[23]), f[25]);
  const T smf3 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(f[1], f[2]), f[7]), f[8]), f[9]), f[10]), f[11]), f[16]), f[20]), f[21]), f[23]), f[25]);
  const T smf4 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(f[3], f[4]), f[7]), f[8]), f[9]), f[10]), f[14]), f[18]), f[20]), f[21]), f[23]), f[25]);
  const T smf5 = rn_add(rn_sub(rn_sub(rn_add(rn_add(rn_add(rn_sub((-f[7]), f[8]), f[9]), f[10]), f[20]), f[21]), f[23]), f[25]);
  const T smf6 = rn_sub(rn_sub(rn_add(rn_add(rn_sub(rn_add(rn_add((-f[7]), f[8]), f[9]), f[10]), f[20]), f[21]), f[23]), f[25]);
  const T smf7 = rn_sub(rn_add(rn_sub(rn_add(rn_sub(rn_add(rn_sub(f[7], f[8]), f[9]), f[10]), f[20]), f[21]), f[23]), f[25]);
  const T smf8 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(f[7], f[8]), f[9]), f[10]), f[20]), f[21]), f[23]), f[25]);
  const T m0 = rho;
  const T m1 = rn_mul(rho, ux);
  const T m2 = rn_mul(rho, uz);
  const T m3 = rn_add(rn_mul((T(1) / T(3)), rho), rn_mul(rn_mul(rho, ux), ux));
  const T m4 = rn_add(rn_mul((T(1) / T(3)), rho), rn_mul(rn_mul(rho, uz), uz));
  const T m5 = rn_mul(rn_mul(rho, ux), uz);
  const T m6 = rn_add(rn_mul(rn_mul((T(1) / T(3)), rho), uz), rn_mul(rn_mul(rn_mul(rho, ux), ux), uz));
  const T m7 = rn_add(rn_mul(rn_mul((T(1) / T(3)), rho), ux), rn_mul(rn_mul(rn_mul(rho, ux), uz), uz));
  const T m8 = rn_add(rn_add(rn_add(rn_mul((T(1) / T(9)), rho), rn_mul(rn_mul(rn_mul((T(1) / T(3)), rho), ux), ux)), rn_mul(rn_mul(rn_mul((T(1) / T(3)), rho), uz), uz)), rn_mul(rn_mul(rn_mul(rn_mul(rho, ux), ux), uz), uz));
  const T s0 = rn_sub(m0, smf0);
  const T s1 = rn_sub(m1, smf1);
  const T s2 = rn_sub(m2, smf2);
  const T s3 = rn_sub(m3, smf3);
  const T s4 = rn_sub(m4, smf4);
  const T s5 = rn_sub(m5, smf5);
  const T s6 = rn_sub(m6, smf6);
  const T s7 = rn_sub(m7, smf7);
  const T s8 = rn_sub(m8, smf8);
  f[6] = rn_add(rn_sub(rn_sub(s0, s3), s4), s8);
  f[12] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), s1), rn_mul((T(1) / T(2)), s3)), rn_mul((T(-1) / T(2)), s7)), rn_mul((T(-1) / T(2)), s8));
  f[13] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(2)), s2), rn_mul((T(1) / T(2)), s4)), rn_mul((T(1) / T(2)), s6)), rn_mul((T(-1) / T(2)), s8));
  f[15] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(2)), s1), rn_mul((T(1) / T(2)), s3)), rn_mul((T(1) / T(2)), s7)), rn_mul((T(-1) / T(2)), s8));
  f[17] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), s2), rn_mul((T(1) / T(2)), s4)), rn_mul((T(-1) / T(2)), s6)), rn_mul((T(-1) / T(2)), s8));
  f[19] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(4)), s5), rn_mul((T(-1) / T(4)), s6)), rn_mul((T(-1) / T(4)), s7)), rn_mul((T(1) / T(4)), s8));
  f[22] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(4)), s5), rn_mul((T(-1) / T(4)), s6)), rn_mul((T(1) / T(4)), s7)), rn_mul((T(1) / T(4)), s8));
  f[24] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(4)), s5), rn_mul((T(1) / T(4)), s6)), rn_mul((T(-1) / T(4)), s7)), rn_mul((T(1) / T(4)), s8));
  f[26] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(4)), s5), rn_mul((T(1) / T(4)), s6)), rn_mul((T(1) / T(4)), s7)), rn_mul((T(1) / T(4)), s8));
}
template <typename T>
PSL_HDI void restore_rho_u_n10(const T (&f)[27], T& rho, T& ux, T& uy, T& uz) {
  const T q0 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_mul((T(3) / T(2)), f[0]), rn_mul((T(3) / T(2)), f[1])), rn_mul((T(3) / T(2)), f[2])), rn_mul((T(3) / T(2)), f[3])), rn_mul((T(3) / T(2)), f[4])), rn_mul((T(3) / T(2)), f[7])), rn_mul((T(3) / T(2)), f[8])), rn_mul((T(3) / T(2)), f[9])), rn_mul((T(3) / T(2)), f[10]));
  const T q1 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_sub(rn_add(rn_sub(rn_add(rn_sub(f[1], f[2]), f[7]), f[8]), f[9]), f[10]), rn_mul(T(-2), f[11])), rn_mul(T(2), f[16])), rn_mul(T(2), f[20])), rn_mul(T(-2), f[21])), rn_mul(T(2), f[23])), rn_mul(T(-2), f[25]));
  const T q2 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), f[0]), rn_mul((T(1) / T(2)), f[1])), rn_mul((T(1) / T(2)), f[2])), rn_mul((T(1) / T(2)), f[3])), rn_mul((T(1) / T(2)), f[4])), rn_mul(T(-2), f[5])), rn_mul((T(1) / T(2)), f[7])), rn_mul((T(1) / T(2)), f[8])), rn_mul((T(1) / T(2)), f[9])), rn_mul((T(1) / T(2)), f[10])), rn_mul(T(-2), f[11])), rn_mul(T(-2), f[14])), rn_mul(T(-2), f[16])), rn_mul(T(-2), f[18])), rn_mul(T(-2), f[20])), rn_mul(T(-2), f[21])), rn_mul(T(-2), f[23])), rn_mul(T(-2), f[25]));
  const T q3 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_sub(rn_add(rn_add(rn_sub(rn_add((-f[3]), f[4]), f[7]), f[8]), f[9]), f[10]), rn_mul(T(2), f[14])), rn_mul(T(-2), f[18])), rn_mul(T(2), f[20])), rn_mul(T(2), f[21])), rn_mul(T(-2), f[23])), rn_mul(T(-2), f[25]));
  rho = q0;
  ux = rn_div(q1, rho);
  uy = rn_div(q2, rho);
  uz = rn_div(q3, rho);
}
template <typename T>
PSL_HDI void restore_u_n10(const T (&f)[27], const T rho, T& ux, T& uy, T& uz) {
  const T scmf0 = rn_div(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_sub(rn_sub(rn_sub(rn_sub(rn_add(rn_sub(rn_sub(rn_sub(rn_sub((-f[0]), f[1]), f[2]), f[3]), f[4]), rn_mul(T(-2), f[5])), f[7]), f[8]), f[9]), f[10]), rn_mul(T(-2), f[11])), rn_mul(T(-2), f[14])), rn_mul(T(-2), f[16])), rn_mul(T(-2), f[18])), rn_mul(T(-2), f[20])), rn_mul(T(-2), f[21])), rn_mul(T(-2), f[23])), rn_mul(T(-2), f[25])), rho);
  const T scmf1 = rn_div(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_sub(rn_sub(rn_add(rn_sub(f[3], f[4]), f[7]), f[8]), f[9]), f[10]), rn_mul(T(-2), f[14])), rn_mul(T(2), f[18])), rn_mul(T(-2), f[20])), rn_mul(T(-2), f[21])), rn_mul(T(2), f[23])), rn_mul(T(2), f[25])), rho);
  const T scmf2 = rn_div(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_sub(rn_add(rn_sub(rn_add((-f[1]), f[2]), f[7]), f[8]), f[9]), f[10]), rn_mul(T(2), f[11])), rn_mul(T(-2), f[16])), rn_mul(T(-2), f[20])), rn_mul(T(2), f[21])), rn_mul(T(-2), f[23])), rn_mul(T(2), f[25])), rho);
  const T s0 = rn_sub(scmf0, T(-1));
  const T s1 = rn_sub(scmf1, T(0));
  const T s2 = rn_sub(scmf2, T(0));
  ux = (-s2);
  uy = s0;
  uz = (-s1);
}
template <typename T>
PSL_HDI void restore_rho_n10(const T (&f)[27], T& rho, const T ux, const T uy, const T uz) {
  const T scqu = rn_mul(T(1), uy);
  const T s = rn_add(T(-1), scqu);
  const T scmf = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_sub(rn_sub(rn_sub(rn_sub(rn_add(rn_sub(rn_sub(rn_sub(rn_sub((-f[0]), f[1]), f[2]), f[3]), f[4]), rn_mul(T(-2), f[5])), f[7]), f[8]), f[9]), f[10]), rn_mul(T(-2), f[11])), rn_mul(T(-2), f[14])), rn_mul(T(-2), f[16])), rn_mul(T(-2), f[18])), rn_mul(T(-2), f[20])), rn_mul(T(-2), f[21])), rn_mul(T(-2), f[23])), rn_mul(T(-2), f[25]));
  rho = rn_div(scmf, s);
}
template <typename T>
PSL_HDI void mirror_n10(T (&f)[27]) {
  f[6] = f[5];
  f[12] = f[16];
  f[13] = f[18];
  f[15] = f[11];
  f[17] = f[14];
  f[19] = f[25];
  f[22] = f[23];
  f[24] = f[21];
  f[26] = f[20];
}

// ---- outer normal (+0,+0,-1): 9 unknown populations ----
template <typename T>
PSL_HDI void mbbc_n12(T (&f)[27], const T rho, const T ux, const T uy, const T uz) {
  const T smf0 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(f[0], f[1]), f[2]), f[3]), f[5]), f[6]), f[7]), f[10]), f[11]), f[12]), f[13]), f[15]), f[16]), f[18]), f[19]), f[22]), f[23]), f[25]);
  const T smf1 = rn_sub(rn_add(rn_add(rn_sub(rn_add(rn_sub(rn_add(rn_sub(rn_sub(rn_add(rn_sub(f[1], f[2]), f[7]), f[10]), f[11]), f[12]), f[15]), f[16]), f[19]), f[22]), f[23]), f[25]);
  const T smf2 = rn_sub(rn_sub(rn_add(rn_add(rn_sub(rn_sub(rn_add(rn_add(rn_add(rn_sub(rn_add((-f[5]), f[6]), f[11]), f[12]), f[13]), f[15]), f[16]), f[18]), f[19]), f[22]), f[23]), f[25]);
  const T smf3 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(f[1], f[2]), f[7]), f[10]), f[11]), f[12]), f[15]), f[16]), f[19]), f[22]), f[23]), f[25]);
  const T smf4 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(f[5], f[6]), f[11]), f[12]), f[13]), f[15]), f[16]), f[18]), f[19]), f[22]), f[23]), f[25]);
  const T smf5 = rn_add(rn_sub(rn_add(rn_sub(rn_sub(rn_sub(rn_add(f[11], f[12]), f[15]), f[16]), f[19]), f[22]), f[23]), f[25]);
  const T smf6 = rn_sub(rn_sub(rn_add(rn_add(rn_sub(rn_add(rn_add((-f[11]), f[12]), f[15]), f[16]), f[19]), f[22]), f[23]), f[25]);
  const T smf7 = rn_sub(rn_add(rn_add(rn_sub(rn_add(rn_sub(rn_add((-f[11]), f[12]), f[15]), f[16]), f[19]), f[22]), f[23]), f[25]);
  const T smf8 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(f[11], f[12]), f[15]), f[16]), f[19]), f[22]), f[23]), f[25]);
  const T m0 = rho;
  const T m1 = rn_mul(rho, ux);
  const T m2 = rn_mul(rho, uy);
  const T m3 = rn_add(rn_mul((T(1) / T(3)), rho), rn_mul(rn_mul(rho, ux), ux));
  const T m4 = rn_add(rn_mul((T(1) / T(3)), rho), rn_mul(rn_mul(rho, uy), uy));
  const T m5 = rn_mul(rn_mul(rho, ux), uy);
  const T m6 = rn_add(rn_mul(rn_mul((T(1) / T(3)), rho), uy), rn_mul(rn_mul(rn_mul(rho, ux), ux), uy));
  const T m7 = rn_add(rn_mul(rn_mul((T(1) / T(3)), rho), ux), rn_mul(rn_mul(rn_mul(rho, ux), uy), uy));
  const T m8 = rn_add(rn_add(rn_add(rn_mul((T(1) / T(9)), rho), rn_mul(rn_mul(rn_mul((T(1) / T(3)), rho), ux), ux)), rn_mul(rn_mul(rn_mul((T(1) / T(3)), rho), uy), uy)), rn_mul(rn_mul(rn_mul(rn_mul(rho, ux), ux), uy), uy));
  const T s0 = rn_sub(m0, smf0);
  const T s1 = rn_sub(m1, smf1);
  const T s2 = rn_sub(m2, smf2);
  const T s3 = rn_sub(m3, smf3);
  const T s4 = rn_sub(m4, smf4);
  const T s5 = rn_sub(m5, smf5);
  const T s6 = rn_sub(m6, smf6);
  const T s7 = rn_sub(m7, smf7);
  const T s8 = rn_sub(m8, smf8);
  f[4] = rn_add(rn_sub(rn_sub(s0, s3), s4), s8);
  f[8] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(2)), s1), rn_mul((T(1) / T(2)), s3)), rn_mul((T(1) / T(2)), s7)), rn_mul((T(-1) / T(2)), s8));
  f[9] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), s1), rn_mul((T(1) / T(2)), s3)), rn_mul((T(-1) / T(2)), s7)), rn_mul((T(-1) / T(2)), s8));
  f[14] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(2)), s2), rn_mul((T(1) / T(2)), s4)), rn_mul((T(1) / T(2)), s6)), rn_mul((T(-1) / T(2)), s8));
  f[17] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), s2), rn_mul((T(1) / T(2)), s4)), rn_mul((T(-1) / T(2)), s6)), rn_mul((T(-1) / T(2)), s8));
  f[20] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(4)), s5), rn_mul((T(-1) / T(4)), s6)), rn_mul((T(1) / T(4)), s7)), rn_mul((T(1) / T(4)), s8));
  f[21] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(4)), s5), rn_mul((T(-1) / T(4)), s6)), rn_mul((T(-1) / T(4)), s7)), rn_mul((T(1) / T(4)), s8));
  f[24] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(4)), s5), rn_mul((T(1) / T(4)), s6)), rn_mul((T(-1) / T(4)), s7)), rn_mul((T(1) / T(4)), s8));
  f[26] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(4)), s5), rn_mul((T(1) / T(4)), s6)), rn_mul((T(1) / T(4)), s7)), rn_mul((T(1) / T(4)), s8));
}
template <typename T>
PSL_HDI void restore_rho_u_n12(const T (&f)[27], T& rho, T& ux, T& uy, T& uz) {
  const T q0 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_mul((T(3) / T(2)), f[0]), rn_mul((T(3) / T(2)), f[1])), rn_mul((T(3) / T(2)), f[2])), rn_mul((T(3) / T(2)), f[5])), rn_mul((T(3) / T(2)), f[6])), rn_mul((T(3) / T(2)), f[11])), rn_mul((T(3) / T(2)), f[12])), rn_mul((T(3) / T(2)), f[15])), rn_mul((T(3) / T(2)), f[16]));
  const T q1 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_sub(rn_add(rn_sub(rn_add(rn_add(rn_sub(f[1], f[2]), rn_mul(T(2), f[7])), rn_mul(T(-2), f[10])), f[11]), f[12]), f[15]), f[16]), rn_mul(T(-2), f[19])), rn_mul(T(2), f[22])), rn_mul(T(2), f[23])), rn_mul(T(-2), f[25]));
  const T q2 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_sub(rn_add(rn_add(rn_add(rn_sub(rn_add((-f[5]), f[6]), f[11]), f[12]), rn_mul(T(2), f[13])), f[15]), f[16]), rn_mul(T(-2), f[18])), rn_mul(T(2), f[19])), rn_mul(T(2), f[22])), rn_mul(T(-2), f[23])), rn_mul(T(-2), f[25]));
  const T q3 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), f[0]), rn_mul((T(1) / T(2)), f[1])), rn_mul((T(1) / T(2)), f[2])), rn_mul(T(-2), f[3])), rn_mul((T(1) / T(2)), f[5])), rn_mul((T(1) / T(2)), f[6])), rn_mul(T(-2), f[7])), rn_mul(T(-2), f[10])), rn_mul((T(1) / T(2)), f[11])), rn_mul((T(1) / T(2)), f[12])), rn_mul(T(-2), f[13])), rn_mul((T(1) / T(2)), f[15])), rn_mul((T(1) / T(2)), f[16])), rn_mul(T(-2), f[18])), rn_mul(T(-2), f[19])), rn_mul(T(-2), f[22])), rn_mul(T(-2), f[23])), rn_mul(T(-2), f[25]));
  rho = q0;
  ux = rn_div(q1, rho);
  uy = rn_div(q2, rho);
  uz = rn_div(q3, rho);
}
template <typename T>
PSL_HDI void restore_u_n12(const T (&f)[27], const T rho, T& ux, T& uy, T& uz) {
  const T scmf0 = rn_div(rn_add(rn_add(rn_add(rn_add(rn_add(rn_sub(rn_sub(rn_add(rn_sub(rn_sub(rn_add(rn_add(rn_sub(rn_sub(rn_add(rn_sub(rn_sub((-f[0]), f[1]), f[2]), rn_mul(T(-2), f[3])), f[5]), f[6]), rn_mul(T(-2), f[7])), rn_mul(T(-2), f[10])), f[11]), f[12]), rn_mul(T(-2), f[13])), f[15]), f[16]), rn_mul(T(-2), f[18])), rn_mul(T(-2), f[19])), rn_mul(T(-2), f[22])), rn_mul(T(-2), f[23])), rn_mul(T(-2), f[25])), rho);
  const T scmf1 = rn_div(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_sub(rn_add(rn_sub(rn_add(rn_sub(f[5], f[6]), f[11]), f[12]), rn_mul(T(-2), f[13])), f[15]), f[16]), rn_mul(T(2), f[18])), rn_mul(T(-2), f[19])), rn_mul(T(-2), f[22])), rn_mul(T(2), f[23])), rn_mul(T(2), f[25])), rho);
  const T scmf2 = rn_div(rn_add(rn_add(rn_add(rn_add(rn_sub(rn_add(rn_sub(rn_add(rn_add(rn_add(rn_add((-f[1]), f[2]), rn_mul(T(-2), f[7])), rn_mul(T(2), f[10])), f[11]), f[12]), f[15]), f[16]), rn_mul(T(2), f[19])), rn_mul(T(-2), f[22])), rn_mul(T(-2), f[23])), rn_mul(T(2), f[25])), rho);
  const T s0 = rn_sub(scmf0, T(-1));
  const T s1 = rn_sub(scmf1, T(0));
  const T s2 = rn_sub(scmf2, T(0));
  ux = (-s2);
  uy = (-s1);
  uz = s0;
}
template <typename T>
PSL_HDI void restore_rho_n12(const T (&f)[27], T& rho, const T ux, const T uy, const T uz) {
  const T scqu = rn_mul(T(1), uz);
  const T s = rn_add(T(-1), scqu);
  const T scmf = rn_add(rn_add(rn_add(rn_add(rn_add(rn_sub(rn_sub(rn_add(rn_sub(rn_sub(rn_add(rn_add(rn_sub(rn_sub(rn_add(rn_sub(rn_sub((-f[0]), f[1]), f[2]), rn_mul(T(-2), f[3])), f[5]), f[6]), rn_mul(T(-2), f[7])), rn_mul(T(-2), f[10])), f[11]), f[12]), rn_mul(T(-2), f[13])), f[15]), f[16]), rn_mul(T(-2), f[18])), rn_mul(T(-2), f[19])), rn_mul(T(-2), f[22])), rn_mul(T(-2), f[23])), rn_mul(T(-2), f[25]));
  rho = rn_div(scmf, s);
}
template <typename T>
PSL_HDI void mirror_n12(T (&f)[27]) {
  f[4] = f[3];
  f[8] = f[10];
  f[9] = f[7];
  f[14] = f[18];
  f[17] = f[13];
  f[20] = f[23];
  f[21] = f[25];
  f[24] = f[19];
  f[26] = f[22];
}

// ---- outer normal (+0,+1,+1): 15 unknown populations ----
template <typename T>
PSL_HDI void mbbc_n17(T (&f)[27], const T rho, const T ux, const T uy, const T uz) {
  const T smf0 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(f[0], f[1]), f[2]), f[4]), f[6]), f[8]), f[9]), f[12]), f[15]), f[17]), f[24]), f[26]);
  const T smf1 = rn_add(rn_sub(rn_sub(rn_add(rn_add(rn_sub(rn_sub(f[1], f[2]), f[8]), f[9]), f[12]), f[15]), f[24]), f[26]);
  const T smf2 = rn_add(rn_add(rn_add(rn_add(rn_add(f[6], f[12]), f[15]), f[17]), f[24]), f[26]);
  const T smf3 = rn_add(rn_add(rn_add(rn_add(rn_add(f[4], f[8]), f[9]), f[17]), f[24]), f[26]);
  const T smf4 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(f[1], f[2]), f[8]), f[9]), f[12]), f[15]), f[24]), f[26]);
  const T smf5 = rn_add(rn_add(rn_add(rn_add(rn_add(f[6], f[12]), f[15]), f[17]), f[24]), f[26]);
  const T smf6 = rn_add(rn_add(rn_add(rn_add(rn_add(f[4], f[8]), f[9]), f[17]), f[24]), f[26]);
  const T smf7 = rn_add(rn_sub(rn_add((-f[8]), f[9]), f[24]), f[26]);
  const T smf8 = rn_add(rn_sub(rn_sub(f[12], f[15]), f[24]), f[26]);
  const T smf9 = rn_add(rn_add(rn_add(f[12], f[15]), f[24]), f[26]);
  const T smf10 = rn_add(rn_add(rn_add(f[8], f[9]), f[24]), f[26]);
  const T smf11 = rn_add(rn_sub(rn_sub(f[12], f[15]), f[24]), f[26]);
  const T smf12 = rn_add(rn_sub(rn_add((-f[8]), f[9]), f[24]), f[26]);
  const T smf13 = rn_add(rn_add(rn_add(f[8], f[9]), f[24]), f[26]);
  const T smf14 = rn_add(rn_add(rn_add(f[12], f[15]), f[24]), f[26]);
  const T m0 = rho;
  const T m1 = rn_mul(rho, ux);
  const T m2 = rn_mul(rho, uy);
  const T m3 = rn_mul(rho, uz);
  const T m4 = rn_add(rn_mul((T(1) / T(3)), rho), rn_mul(rn_mul(rho, ux), ux));
  const T m5 = rn_add(rn_mul((T(1) / T(3)), rho), rn_mul(rn_mul(rho, uy), uy));
  const T m6 = rn_add(rn_mul((T(1) / T(3)), rho), rn_mul(rn_mul(rho, uz), uz));
  const T m7 = rn_mul(rn_mul(rho, ux), uz);
  const T m8 = rn_mul(rn_mul(rho, ux), uy);
  const T m9 = rn_add(rn_mul(rn_mul((T(1) / T(3)), rho), uy), rn_mul(rn_mul(rn_mul(rho, ux), ux), uy));
  const T m10 = rn_add(rn_mul(rn_mul((T(1) / T(3)), rho), uz), rn_mul(rn_mul(rn_mul(rho, ux), ux), uz));
  const T m11 = rn_add(rn_mul(rn_mul((T(1) / T(3)), rho), ux), rn_mul(rn_mul(rn_mul(rho, ux), uy), uy));
  const T m12 = rn_add(rn_mul(rn_mul((T(1) / T(3)), rho), ux), rn_mul(rn_mul(rn_mul(rho, ux), uz), uz));
  const T m13 = rn_add(rn_add(rn_add(rn_mul((T(1) / T(9)), rho), rn_mul(rn_mul(rn_mul((T(1) / T(3)), rho), ux), ux)), rn_mul(rn_mul(rn_mul((T(1) / T(3)), rho), uz), uz)), rn_mul(rn_mul(rn_mul(rn_mul(rho, ux), ux), uz), uz));
  const T m14 = rn_add(rn_add(rn_add(rn_mul((T(1) / T(9)), rho), rn_mul(rn_mul(rn_mul((T(1) / T(3)), rho), ux), ux)), rn_mul(rn_mul(rn_mul((T(1) / T(3)), rho), uy), uy)), rn_mul(rn_mul(rn_mul(rn_mul(rho, ux), ux), uy), uy));
  const T s0 = rn_sub(m0, smf0);
  const T s1 = rn_sub(m1, smf1);
  const T s2 = rn_sub(m2, smf2);
  const T s3 = rn_sub(m3, smf3);
  const T s4 = rn_sub(m4, smf4);
  const T s5 = rn_sub(m5, smf5);
  const T s6 = rn_sub(m6, smf6);
  const T s7 = rn_sub(m7, smf7);
  const T s8 = rn_sub(m8, smf8);
  const T s9 = rn_sub(m9, smf9);
  const T s10 = rn_sub(m10, smf10);
  const T s11 = rn_sub(m11, smf11);
  const T s12 = rn_sub(m12, smf12);
  const T s13 = rn_sub(m13, smf13);
  const T s14 = rn_sub(m14, smf14);
  f[3] = rn_add(rn_sub(rn_sub(s0, s4), s5), s14);
  f[5] = rn_add(rn_sub(rn_sub(s0, s4), s6), s13);
  f[7] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), s1), rn_mul((T(1) / T(2)), s4)), rn_mul((T(-1) / T(2)), s11)), rn_mul((T(-1) / T(2)), s14));
  f[10] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(2)), s1), rn_mul((T(1) / T(2)), s4)), rn_mul((T(1) / T(2)), s11)), rn_mul((T(-1) / T(2)), s14));
  f[11] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(2)), s1), rn_mul((T(1) / T(2)), s4)), rn_mul((T(1) / T(2)), s12)), rn_mul((T(-1) / T(2)), s13));
  f[13] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), s2), rn_mul((T(1) / T(2)), s5)), rn_mul((T(-1) / T(2)), s9)), rn_mul((T(-1) / T(2)), s14));
  f[14] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), s3), rn_mul((T(1) / T(2)), s6)), rn_mul((T(-1) / T(2)), s10)), rn_mul((T(-1) / T(2)), s13));
  f[16] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), s1), rn_mul((T(1) / T(2)), s4)), rn_mul((T(-1) / T(2)), s12)), rn_mul((T(-1) / T(2)), s13));
  f[18] = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add((-s0), rn_mul((T(-1) / T(2)), s2)), rn_mul((T(-1) / T(2)), s3)), s4), rn_mul((T(1) / T(2)), s5)), rn_mul((T(1) / T(2)), s6)), rn_mul((T(1) / T(2)), s9)), rn_mul((T(1) / T(2)), s10)), rn_mul((T(-1) / T(2)), s13)), rn_mul((T(-1) / T(2)), s14));
  f[19] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(4)), s8), rn_mul((T(1) / T(4)), s9)), rn_mul((T(-1) / T(4)), s11)), rn_mul((T(1) / T(4)), s14));
  f[20] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(4)), s7), rn_mul((T(1) / T(4)), s10)), rn_mul((T(1) / T(4)), s12)), rn_mul((T(1) / T(4)), s13));
  f[21] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(4)), s7), rn_mul((T(1) / T(4)), s10)), rn_mul((T(-1) / T(4)), s12)), rn_mul((T(1) / T(4)), s13));
  f[22] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(4)), s8), rn_mul((T(1) / T(4)), s9)), rn_mul((T(1) / T(4)), s11)), rn_mul((T(1) / T(4)), s14));
  f[23] = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_mul((T(-1) / T(2)), s1), rn_mul((T(-1) / T(2)), s4)), rn_mul((T(-1) / T(4)), s7)), rn_mul((T(-1) / T(4)), s8)), rn_mul((T(-1) / T(4)), s9)), rn_mul((T(-1) / T(4)), s10)), rn_mul((T(1) / T(4)), s11)), rn_mul((T(1) / T(4)), s12)), rn_mul((T(1) / T(4)), s13)), rn_mul((T(1) / T(4)), s14));
  f[25] = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), s1), rn_mul((T(-1) / T(2)), s4)), rn_mul((T(1) / T(4)), s7)), rn_mul((T(1) / T(4)), s8)), rn_mul((T(-1) / T(4)), s9)), rn_mul((T(-1) / T(4)), s10)), rn_mul((T(-1) / T(4)), s11)), rn_mul((T(-1) / T(4)), s12)), rn_mul((T(1) / T(4)), s13)), rn_mul((T(1) / T(4)), s14));
}
template <typename T>
PSL_HDI void restore_rho_u_n17(const T (&f)[27], T& rho, T& ux, T& uy, T& uz) {
  const T q0 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_mul(T(2), f[0]), rn_mul(T(2), f[1])), rn_mul(T(2), f[2])), f[4]), f[6]), f[8]), f[9]), f[12]), f[15]), rn_mul(T(-4), f[17])), rn_mul(T(-4), f[24])), rn_mul(T(-4), f[26]));
  const T q1 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_sub(f[1], f[2]), rn_mul(T(-2), f[8])), rn_mul(T(2), f[9])), rn_mul(T(2), f[12])), rn_mul(T(-2), f[15])), rn_mul(T(-4), f[24])), rn_mul(T(4), f[26]));
  const T q2 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_sub(rn_sub(rn_add(rn_sub(rn_add(rn_add(rn_mul((T(-1) / T(2)), f[0]), rn_mul((T(-1) / T(2)), f[1])), rn_mul((T(-1) / T(2)), f[2])), f[4]), rn_mul(T(2), f[6])), f[8]), f[9]), rn_mul(T(2), f[12])), rn_mul(T(2), f[15])), rn_mul(T(4), f[17])), rn_mul(T(4), f[24])), rn_mul(T(4), f[26]));
  const T q3 = rn_add(rn_add(rn_add(rn_sub(rn_sub(rn_add(rn_add(rn_sub(rn_add(rn_add(rn_add(rn_mul((T(-1) / T(2)), f[0]), rn_mul((T(-1) / T(2)), f[1])), rn_mul((T(-1) / T(2)), f[2])), rn_mul(T(2), f[4])), f[6]), rn_mul(T(2), f[8])), rn_mul(T(2), f[9])), f[12]), f[15]), rn_mul(T(4), f[17])), rn_mul(T(4), f[24])), rn_mul(T(4), f[26]));
  rho = q0;
  ux = rn_div(q1, rho);
  uy = rn_div(q2, rho);
  uz = rn_div(q3, rho);
}
template <typename T>
PSL_HDI void restore_u_n17(const T (&f)[27], const T rho, T& ux, T& uy, T& uz) {
  const T scmf0 = rn_div(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(f[0], f[1]), f[2]), rn_mul(T(2), f[4])), rn_mul(T(2), f[6])), rn_mul(T(2), f[8])), rn_mul(T(2), f[9])), rn_mul(T(2), f[12])), rn_mul(T(2), f[15])), rn_mul(T(4), f[17])), rn_mul(T(4), f[24])), rn_mul(T(4), f[26])), rho);
  const T scmf1 = rn_div(rn_add(rn_add(rn_add(rn_sub(rn_sub((-f[0]), f[1]), f[2]), rn_mul(T(-2), f[4])), rn_mul(T(-2), f[8])), rn_mul(T(-2), f[9])), rho);
  const T scmf2 = rn_div(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_sub(f[1], f[2]), rn_mul(T(-2), f[8])), rn_mul(T(2), f[9])), rn_mul(T(2), f[12])), rn_mul(T(-2), f[15])), rn_mul(T(-4), f[24])), rn_mul(T(4), f[26])), rho);
  const T s0 = rn_sub(scmf0, T(1));
  const T s1 = rn_sub(scmf1, (T(-2) / T(3)));
  const T s2 = rn_sub(scmf2, T(0));
  ux = s2;
  uy = rn_add(s0, rn_mul((T(3) / T(2)), s1));
  uz = rn_mul((T(-3) / T(2)), s1);
}
template <typename T>
PSL_HDI void restore_rho_n17(const T (&f)[27], T& rho, const T ux, const T uy, const T uz) {
  const T scqu = rn_add(rn_mul(T(1), uy), rn_mul(T(1), uz));
  const T s = rn_add(T(1), scqu);
  const T scmf = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(f[0], f[1]), f[2]), rn_mul(T(2), f[4])), rn_mul(T(2), f[6])), rn_mul(T(2), f[8])), rn_mul(T(2), f[9])), rn_mul(T(2), f[12])), rn_mul(T(2), f[15])), rn_mul(T(4), f[17])), rn_mul(T(4), f[24])), rn_mul(T(4), f[26]));
  rho = rn_div(scmf, s);
}
template <typename T>
PSL_HDI void mirror_n17(T (&f)[27]) {
  f[3] = f[4];
  f[5] = f[6];
  f[7] = f[9];
  f[10] = f[8];
  f[11] = f[15];
  f[13] = f[17];
  f[14] = f[17];
  f[16] = f[12];
  f[18] = f[17];
  f[19] = f[24];
  f[20] = f[26];
  f[21] = f[24];
  f[22] = f[26];
  f[23] = f[26];
  f[25] = f[24];
}

// ---- outer normal (+1,+0,+1): 15 unknown populations ----
template <typename T>
PSL_HDI void mbbc_n23(T (&f)[27], const T rho, const T ux, const T uy, const T uz) {
  const T smf0 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(f[0], f[1]), f[4]), f[5]), f[6]), f[9]), f[12]), f[14]), f[16]), f[17]), f[20]), f[26]);
  const T smf1 = rn_add(rn_add(rn_add(rn_add(rn_add(f[1], f[9]), f[12]), f[16]), f[20]), f[26]);
  const T smf2 = rn_add(rn_sub(rn_add(rn_sub(rn_sub(rn_add(rn_add((-f[5]), f[6]), f[12]), f[14]), f[16]), f[17]), f[20]), f[26]);
  const T smf3 = rn_add(rn_add(rn_add(rn_add(rn_add(f[4], f[9]), f[14]), f[17]), f[20]), f[26]);
  const T smf4 = rn_add(rn_add(rn_add(rn_add(rn_add(f[1], f[9]), f[12]), f[16]), f[20]), f[26]);
  const T smf5 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(f[5], f[6]), f[12]), f[14]), f[16]), f[17]), f[20]), f[26]);
  const T smf6 = rn_add(rn_add(rn_add(rn_add(rn_add(f[4], f[9]), f[14]), f[17]), f[20]), f[26]);
  const T smf7 = rn_add(rn_sub(rn_add((-f[14]), f[17]), f[20]), f[26]);
  const T smf8 = rn_add(rn_sub(rn_sub(f[12], f[16]), f[20]), f[26]);
  const T smf9 = rn_add(rn_sub(rn_sub(f[12], f[16]), f[20]), f[26]);
  const T smf10 = rn_add(rn_add(rn_add(f[12], f[16]), f[20]), f[26]);
  const T smf11 = rn_add(rn_add(rn_add(f[14], f[17]), f[20]), f[26]);
  const T smf12 = rn_add(rn_sub(rn_add((-f[14]), f[17]), f[20]), f[26]);
  const T smf13 = rn_add(rn_add(rn_add(f[14], f[17]), f[20]), f[26]);
  const T smf14 = rn_add(rn_add(rn_add(f[12], f[16]), f[20]), f[26]);
  const T m0 = rho;
  const T m1 = rn_mul(rho, ux);
  const T m2 = rn_mul(rho, uy);
  const T m3 = rn_mul(rho, uz);
  const T m4 = rn_add(rn_mul((T(1) / T(3)), rho), rn_mul(rn_mul(rho, ux), ux));
  const T m5 = rn_add(rn_mul((T(1) / T(3)), rho), rn_mul(rn_mul(rho, uy), uy));
  const T m6 = rn_add(rn_mul((T(1) / T(3)), rho), rn_mul(rn_mul(rho, uz), uz));
  const T m7 = rn_mul(rn_mul(rho, uy), uz);
  const T m8 = rn_mul(rn_mul(rho, ux), uy);
  const T m9 = rn_add(rn_mul(rn_mul((T(1) / T(3)), rho), uy), rn_mul(rn_mul(rn_mul(rho, ux), ux), uy));
  const T m10 = rn_add(rn_mul(rn_mul((T(1) / T(3)), rho), ux), rn_mul(rn_mul(rn_mul(rho, ux), uy), uy));
  const T m11 = rn_add(rn_mul(rn_mul((T(1) / T(3)), rho), uz), rn_mul(rn_mul(rn_mul(rho, uy), uy), uz));
  const T m12 = rn_add(rn_mul(rn_mul((T(1) / T(3)), rho), uy), rn_mul(rn_mul(rn_mul(rho, uy), uz), uz));
  const T m13 = rn_add(rn_add(rn_add(rn_mul((T(1) / T(9)), rho), rn_mul(rn_mul(rn_mul((T(1) / T(3)), rho), uy), uy)), rn_mul(rn_mul(rn_mul((T(1) / T(3)), rho), uz), uz)), rn_mul(rn_mul(rn_mul(rn_mul(rho, uy), uy), uz), uz));
  const T m14 = rn_add(rn_add(rn_add(rn_mul((T(1) / T(9)), rho), rn_mul(rn_mul(rn_mul((T(1) / T(3)), rho), ux), ux)), rn_mul(rn_mul(rn_mul((T(1) / T(3)), rho), uy), uy)), rn_mul(rn_mul(rn_mul(rn_mul(rho, ux), ux), uy), uy));
  const T s0 = rn_sub(m0, smf0);
  const T s1 = rn_sub(m1, smf1);
  const T s2 = rn_sub(m2, smf2);
  const T s3 = rn_sub(m3, smf3);
  const T s4 = rn_sub(m4, smf4);
  const T s5 = rn_sub(m5, smf5);
  const T s6 = rn_sub(m6, smf6);
  const T s7 = rn_sub(m7, smf7);
  const T s8 = rn_sub(m8, smf8);
  const T s9 = rn_sub(m9, smf9);
  const T s10 = rn_sub(m10, smf10);
  const T s11 = rn_sub(m11, smf11);
  const T s12 = rn_sub(m12, smf12);
  const T s13 = rn_sub(m13, smf13);
  const T s14 = rn_sub(m14, smf14);
  f[2] = rn_add(rn_sub(rn_sub(s0, s5), s6), s13);
  f[3] = rn_add(rn_sub(rn_sub(s0, s4), s5), s14);
  f[7] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), s1), rn_mul((T(1) / T(2)), s4)), rn_mul((T(-1) / T(2)), s10)), rn_mul((T(-1) / T(2)), s14));
  f[8] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), s3), rn_mul((T(1) / T(2)), s6)), rn_mul((T(-1) / T(2)), s11)), rn_mul((T(-1) / T(2)), s13));
  f[10] = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add((-s0), rn_mul((T(-1) / T(2)), s1)), rn_mul((T(-1) / T(2)), s3)), rn_mul((T(1) / T(2)), s4)), s5), rn_mul((T(1) / T(2)), s6)), rn_mul((T(1) / T(2)), s10)), rn_mul((T(1) / T(2)), s11)), rn_mul((T(-1) / T(2)), s13)), rn_mul((T(-1) / T(2)), s14));
  f[11] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(2)), s2), rn_mul((T(1) / T(2)), s5)), rn_mul((T(1) / T(2)), s12)), rn_mul((T(-1) / T(2)), s13));
  f[13] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), s2), rn_mul((T(1) / T(2)), s5)), rn_mul((T(-1) / T(2)), s9)), rn_mul((T(-1) / T(2)), s14));
  f[15] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), s2), rn_mul((T(1) / T(2)), s5)), rn_mul((T(-1) / T(2)), s12)), rn_mul((T(-1) / T(2)), s13));
  f[18] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(2)), s2), rn_mul((T(1) / T(2)), s5)), rn_mul((T(1) / T(2)), s9)), rn_mul((T(-1) / T(2)), s14));
  f[19] = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_mul((T(-1) / T(2)), s2), rn_mul((T(-1) / T(2)), s5)), rn_mul((T(-1) / T(4)), s7)), rn_mul((T(-1) / T(4)), s8)), rn_mul((T(1) / T(4)), s9)), rn_mul((T(-1) / T(4)), s10)), rn_mul((T(-1) / T(4)), s11)), rn_mul((T(1) / T(4)), s12)), rn_mul((T(1) / T(4)), s13)), rn_mul((T(1) / T(4)), s14));
  f[21] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(4)), s7), rn_mul((T(1) / T(4)), s11)), rn_mul((T(-1) / T(4)), s12)), rn_mul((T(1) / T(4)), s13));
  f[22] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(4)), s8), rn_mul((T(1) / T(4)), s9)), rn_mul((T(1) / T(4)), s10)), rn_mul((T(1) / T(4)), s14));
  f[23] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(4)), s8), rn_mul((T(-1) / T(4)), s9)), rn_mul((T(1) / T(4)), s10)), rn_mul((T(1) / T(4)), s14));
  f[24] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(4)), s7), rn_mul((T(1) / T(4)), s11)), rn_mul((T(1) / T(4)), s12)), rn_mul((T(1) / T(4)), s13));
  f[25] = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), s2), rn_mul((T(-1) / T(2)), s5)), rn_mul((T(1) / T(4)), s7)), rn_mul((T(1) / T(4)), s8)), rn_mul((T(-1) / T(4)), s9)), rn_mul((T(-1) / T(4)), s10)), rn_mul((T(-1) / T(4)), s11)), rn_mul((T(-1) / T(4)), s12)), rn_mul((T(1) / T(4)), s13)), rn_mul((T(1) / T(4)), s14));
}
template <typename T>
PSL_HDI void restore_rho_u_n23(const T (&f)[27], T& rho, T& ux, T& uy, T& uz) {
  const T q0 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_mul(T(2), f[0]), f[1]), f[4]), rn_mul(T(2), f[5])), rn_mul(T(2), f[6])), rn_mul(T(-4), f[9])), f[12]), f[14]), f[16]), f[17]), rn_mul(T(-4), f[20])), rn_mul(T(-4), f[26]));
  const T q1 = rn_add(rn_add(rn_sub(rn_add(rn_sub(rn_add(rn_add(rn_add(rn_add(rn_sub(rn_add(rn_mul((T(-1) / T(2)), f[0]), rn_mul(T(2), f[1])), f[4]), rn_mul((T(-1) / T(2)), f[5])), rn_mul((T(-1) / T(2)), f[6])), rn_mul(T(4), f[9])), rn_mul(T(2), f[12])), f[14]), rn_mul(T(2), f[16])), f[17]), rn_mul(T(4), f[20])), rn_mul(T(4), f[26]));
  const T q2 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add((-f[5]), f[6]), rn_mul(T(2), f[12])), rn_mul(T(-2), f[14])), rn_mul(T(-2), f[16])), rn_mul(T(2), f[17])), rn_mul(T(-4), f[20])), rn_mul(T(4), f[26]));
  const T q3 = rn_add(rn_add(rn_add(rn_sub(rn_add(rn_sub(rn_add(rn_add(rn_add(rn_add(rn_sub(rn_mul((T(-1) / T(2)), f[0]), f[1]), rn_mul(T(2), f[4])), rn_mul((T(-1) / T(2)), f[5])), rn_mul((T(-1) / T(2)), f[6])), rn_mul(T(4), f[9])), f[12]), rn_mul(T(2), f[14])), f[16]), rn_mul(T(2), f[17])), rn_mul(T(4), f[20])), rn_mul(T(4), f[26]));
  rho = q0;
  ux = rn_div(q1, rho);
  uy = rn_div(q2, rho);
  uz = rn_div(q3, rho);
}
template <typename T>
PSL_HDI void restore_u_n23(const T (&f)[27], const T rho, T& ux, T& uy, T& uz) {
  const T scmf0 = rn_div(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(f[0], rn_mul(T(2), f[1])), rn_mul(T(2), f[4])), f[5]), f[6]), rn_mul(T(4), f[9])), rn_mul(T(2), f[12])), rn_mul(T(2), f[14])), rn_mul(T(2), f[16])), rn_mul(T(2), f[17])), rn_mul(T(4), f[20])), rn_mul(T(4), f[26])), rho);
  const T scmf1 = rn_div(rn_add(rn_add(rn_sub(rn_sub(rn_add((-f[0]), rn_mul(T(-2), f[4])), f[5]), f[6]), rn_mul(T(-2), f[14])), rn_mul(T(-2), f[17])), rho);
  const T scmf2 = rn_div(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add((-f[5]), f[6]), rn_mul(T(2), f[12])), rn_mul(T(-2), f[14])), rn_mul(T(-2), f[16])), rn_mul(T(2), f[17])), rn_mul(T(-4), f[20])), rn_mul(T(4), f[26])), rho);
  const T s0 = rn_sub(scmf0, T(1));
  const T s1 = rn_sub(scmf1, (T(-2) / T(3)));
  const T s2 = rn_sub(scmf2, T(0));
  ux = rn_add(s0, rn_mul((T(3) / T(2)), s1));
  uy = s2;
  uz = rn_mul((T(-3) / T(2)), s1);
}
template <typename T>
PSL_HDI void restore_rho_n23(const T (&f)[27], T& rho, const T ux, const T uy, const T uz) {
  const T scqu = rn_add(rn_mul(T(1), ux), rn_mul(T(1), uz));
  const T s = rn_add(T(1), scqu);
  const T scmf = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(f[0], rn_mul(T(2), f[1])), rn_mul(T(2), f[4])), f[5]), f[6]), rn_mul(T(4), f[9])), rn_mul(T(2), f[12])), rn_mul(T(2), f[14])), rn_mul(T(2), f[16])), rn_mul(T(2), f[17])), rn_mul(T(4), f[20])), rn_mul(T(4), f[26]));
  rho = rn_div(scmf, s);
}
template <typename T>
PSL_HDI void mirror_n23(T (&f)[27]) {
  f[2] = f[1];
  f[3] = f[4];
  f[7] = f[9];
  f[8] = f[9];
  f[10] = f[9];
  f[11] = f[16];
  f[13] = f[17];
  f[15] = f[12];
  f[18] = f[14];
  f[19] = f[26];
  f[21] = f[20];
  f[22] = f[26];
  f[23] = f[20];
  f[24] = f[26];
  f[25] = f[20];
}

// ---- outer normal (+1,+1,+0): 15 unknown populations ----
template <typename T>
PSL_HDI void mbbc_n25(T (&f)[27], const T rho, const T ux, const T uy, const T uz) {
  const T smf0 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(f[0], f[1]), f[3]), f[4]), f[6]), f[7]), f[9]), f[12]), f[13]), f[17]), f[22]), f[26]);
  const T smf1 = rn_add(rn_add(rn_add(rn_add(rn_add(f[1], f[7]), f[9]), f[12]), f[22]), f[26]);
  const T smf2 = rn_add(rn_add(rn_add(rn_add(rn_add(f[6], f[12]), f[13]), f[17]), f[22]), f[26]);
  const T smf3 = rn_add(rn_sub(rn_add(rn_sub(rn_add(rn_sub(rn_add((-f[3]), f[4]), f[7]), f[9]), f[13]), f[17]), f[22]), f[26]);
  const T smf4 = rn_add(rn_add(rn_add(rn_add(rn_add(f[1], f[7]), f[9]), f[12]), f[22]), f[26]);
  const T smf5 = rn_add(rn_add(rn_add(rn_add(rn_add(f[6], f[12]), f[13]), f[17]), f[22]), f[26]);
  const T smf6 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(f[3], f[4]), f[7]), f[9]), f[13]), f[17]), f[22]), f[26]);
  const T smf7 = rn_add(rn_sub(rn_add((-f[13]), f[17]), f[22]), f[26]);
  const T smf8 = rn_add(rn_sub(rn_add((-f[7]), f[9]), f[22]), f[26]);
  const T smf9 = rn_add(rn_sub(rn_add((-f[7]), f[9]), f[22]), f[26]);
  const T smf10 = rn_add(rn_sub(rn_add((-f[13]), f[17]), f[22]), f[26]);
  const T smf11 = rn_add(rn_add(rn_add(f[7], f[9]), f[22]), f[26]);
  const T smf12 = rn_add(rn_add(rn_add(f[13], f[17]), f[22]), f[26]);
  const T smf13 = rn_add(rn_add(rn_add(f[13], f[17]), f[22]), f[26]);
  const T smf14 = rn_add(rn_add(rn_add(f[7], f[9]), f[22]), f[26]);
  const T m0 = rho;
  const T m1 = rn_mul(rho, ux);
  const T m2 = rn_mul(rho, uy);
  const T m3 = rn_mul(rho, uz);
  const T m4 = rn_add(rn_mul((T(1) / T(3)), rho), rn_mul(rn_mul(rho, ux), ux));
  const T m5 = rn_add(rn_mul((T(1) / T(3)), rho), rn_mul(rn_mul(rho, uy), uy));
  const T m6 = rn_add(rn_mul((T(1) / T(3)), rho), rn_mul(rn_mul(rho, uz), uz));
  const T m7 = rn_mul(rn_mul(rho, uy), uz);
  const T m8 = rn_mul(rn_mul(rho, ux), uz);
  const T m9 = rn_add(rn_mul(rn_mul((T(1) / T(3)), rho), uz), rn_mul(rn_mul(rn_mul(rho, ux), ux), uz));
  const T m10 = rn_add(rn_mul(rn_mul((T(1) / T(3)), rho), uz), rn_mul(rn_mul(rn_mul(rho, uy), uy), uz));
  const T m11 = rn_add(rn_mul(rn_mul((T(1) / T(3)), rho), ux), rn_mul(rn_mul(rn_mul(rho, ux), uz), uz));
  const T m12 = rn_add(rn_mul(rn_mul((T(1) / T(3)), rho), uy), rn_mul(rn_mul(rn_mul(rho, uy), uz), uz));
  const T m13 = rn_add(rn_add(rn_add(rn_mul((T(1) / T(9)), rho), rn_mul(rn_mul(rn_mul((T(1) / T(3)), rho), uy), uy)), rn_mul(rn_mul(rn_mul((T(1) / T(3)), rho), uz), uz)), rn_mul(rn_mul(rn_mul(rn_mul(rho, uy), uy), uz), uz));
  const T m14 = rn_add(rn_add(rn_add(rn_mul((T(1) / T(9)), rho), rn_mul(rn_mul(rn_mul((T(1) / T(3)), rho), ux), ux)), rn_mul(rn_mul(rn_mul((T(1) / T(3)), rho), uz), uz)), rn_mul(rn_mul(rn_mul(rn_mul(rho, ux), ux), uz), uz));
  const T s0 = rn_sub(m0, smf0);
  const T s1 = rn_sub(m1, smf1);
  const T s2 = rn_sub(m2, smf2);
  const T s3 = rn_sub(m3, smf3);
  const T s4 = rn_sub(m4, smf4);
  const T s5 = rn_sub(m5, smf5);
  const T s6 = rn_sub(m6, smf6);
  const T s7 = rn_sub(m7, smf7);
  const T s8 = rn_sub(m8, smf8);
  const T s9 = rn_sub(m9, smf9);
  const T s10 = rn_sub(m10, smf10);
  const T s11 = rn_sub(m11, smf11);
  const T s12 = rn_sub(m12, smf12);
  const T s13 = rn_sub(m13, smf13);
  const T s14 = rn_sub(m14, smf14);
  f[2] = rn_add(rn_sub(rn_sub(s0, s5), s6), s13);
  f[5] = rn_add(rn_sub(rn_sub(s0, s4), s6), s14);
  f[8] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), s3), rn_mul((T(1) / T(2)), s6)), rn_mul((T(-1) / T(2)), s10)), rn_mul((T(-1) / T(2)), s13));
  f[10] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(2)), s3), rn_mul((T(1) / T(2)), s6)), rn_mul((T(1) / T(2)), s10)), rn_mul((T(-1) / T(2)), s13));
  f[11] = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add((-s0), rn_mul((T(-1) / T(2)), s1)), rn_mul((T(-1) / T(2)), s2)), rn_mul((T(1) / T(2)), s4)), rn_mul((T(1) / T(2)), s5)), s6), rn_mul((T(1) / T(2)), s11)), rn_mul((T(1) / T(2)), s12)), rn_mul((T(-1) / T(2)), s13)), rn_mul((T(-1) / T(2)), s14));
  f[14] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), s3), rn_mul((T(1) / T(2)), s6)), rn_mul((T(-1) / T(2)), s9)), rn_mul((T(-1) / T(2)), s14));
  f[15] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), s2), rn_mul((T(1) / T(2)), s5)), rn_mul((T(-1) / T(2)), s12)), rn_mul((T(-1) / T(2)), s13));
  f[16] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), s1), rn_mul((T(1) / T(2)), s4)), rn_mul((T(-1) / T(2)), s11)), rn_mul((T(-1) / T(2)), s14));
  f[18] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(2)), s3), rn_mul((T(1) / T(2)), s6)), rn_mul((T(1) / T(2)), s9)), rn_mul((T(-1) / T(2)), s14));
  f[19] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(4)), s7), rn_mul((T(-1) / T(4)), s10)), rn_mul((T(1) / T(4)), s12)), rn_mul((T(1) / T(4)), s13));
  f[20] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(4)), s8), rn_mul((T(1) / T(4)), s9)), rn_mul((T(1) / T(4)), s11)), rn_mul((T(1) / T(4)), s14));
  f[21] = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_mul((T(-1) / T(2)), s3), rn_mul((T(-1) / T(2)), s6)), rn_mul((T(-1) / T(4)), s7)), rn_mul((T(-1) / T(4)), s8)), rn_mul((T(1) / T(4)), s9)), rn_mul((T(1) / T(4)), s10)), rn_mul((T(-1) / T(4)), s11)), rn_mul((T(-1) / T(4)), s12)), rn_mul((T(1) / T(4)), s13)), rn_mul((T(1) / T(4)), s14));
  f[23] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(4)), s8), rn_mul((T(-1) / T(4)), s9)), rn_mul((T(1) / T(4)), s11)), rn_mul((T(1) / T(4)), s14));
  f[24] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(4)), s7), rn_mul((T(1) / T(4)), s10)), rn_mul((T(1) / T(4)), s12)), rn_mul((T(1) / T(4)), s13));
  f[25] = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), s3), rn_mul((T(-1) / T(2)), s6)), rn_mul((T(1) / T(4)), s7)), rn_mul((T(1) / T(4)), s8)), rn_mul((T(-1) / T(4)), s9)), rn_mul((T(-1) / T(4)), s10)), rn_mul((T(-1) / T(4)), s11)), rn_mul((T(-1) / T(4)), s12)), rn_mul((T(1) / T(4)), s13)), rn_mul((T(1) / T(4)), s14));
}
template <typename T>
PSL_HDI void restore_rho_u_n25(const T (&f)[27], T& rho, T& ux, T& uy, T& uz) {
  const T q0 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_mul(T(2), f[0]), f[1]), rn_mul(T(2), f[3])), rn_mul(T(2), f[4])), f[6]), f[7]), f[9]), rn_mul(T(-4), f[12])), f[13]), f[17]), rn_mul(T(-4), f[22])), rn_mul(T(-4), f[26]));
  const T q1 = rn_add(rn_add(rn_sub(rn_sub(rn_add(rn_add(rn_add(rn_sub(rn_add(rn_add(rn_add(rn_mul((T(-1) / T(2)), f[0]), rn_mul(T(2), f[1])), rn_mul((T(-1) / T(2)), f[3])), rn_mul((T(-1) / T(2)), f[4])), f[6]), rn_mul(T(2), f[7])), rn_mul(T(2), f[9])), rn_mul(T(4), f[12])), f[13]), f[17]), rn_mul(T(4), f[22])), rn_mul(T(4), f[26]));
  const T q2 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_sub(rn_sub(rn_add(rn_add(rn_add(rn_sub(rn_mul((T(-1) / T(2)), f[0]), f[1]), rn_mul((T(-1) / T(2)), f[3])), rn_mul((T(-1) / T(2)), f[4])), rn_mul(T(2), f[6])), f[7]), f[9]), rn_mul(T(4), f[12])), rn_mul(T(2), f[13])), rn_mul(T(2), f[17])), rn_mul(T(4), f[22])), rn_mul(T(4), f[26]));
  const T q3 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add((-f[3]), f[4]), rn_mul(T(-2), f[7])), rn_mul(T(2), f[9])), rn_mul(T(-2), f[13])), rn_mul(T(2), f[17])), rn_mul(T(-4), f[22])), rn_mul(T(4), f[26]));
  rho = q0;
  ux = rn_div(q1, rho);
  uy = rn_div(q2, rho);
  uz = rn_div(q3, rho);
}
template <typename T>
PSL_HDI void restore_u_n25(const T (&f)[27], const T rho, T& ux, T& uy, T& uz) {
  const T scmf0 = rn_div(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(f[0], rn_mul(T(2), f[1])), f[3]), f[4]), rn_mul(T(2), f[6])), rn_mul(T(2), f[7])), rn_mul(T(2), f[9])), rn_mul(T(4), f[12])), rn_mul(T(2), f[13])), rn_mul(T(2), f[17])), rn_mul(T(4), f[22])), rn_mul(T(4), f[26])), rho);
  const T scmf1 = rn_div(rn_add(rn_add(rn_add(rn_sub(rn_sub((-f[0]), f[3]), f[4]), rn_mul(T(-2), f[6])), rn_mul(T(-2), f[13])), rn_mul(T(-2), f[17])), rho);
  const T scmf2 = rn_div(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add((-f[3]), f[4]), rn_mul(T(-2), f[7])), rn_mul(T(2), f[9])), rn_mul(T(-2), f[13])), rn_mul(T(2), f[17])), rn_mul(T(-4), f[22])), rn_mul(T(4), f[26])), rho);
  const T s0 = rn_sub(scmf0, T(1));
  const T s1 = rn_sub(scmf1, (T(-2) / T(3)));
  const T s2 = rn_sub(scmf2, T(0));
  ux = rn_add(s0, rn_mul((T(3) / T(2)), s1));
  uy = rn_mul((T(-3) / T(2)), s1);
  uz = s2;
}
template <typename T>
PSL_HDI void restore_rho_n25(const T (&f)[27], T& rho, const T ux, const T uy, const T uz) {
  const T scqu = rn_add(rn_mul(T(1), ux), rn_mul(T(1), uy));
  const T s = rn_add(T(1), scqu);
  const T scmf = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(f[0], rn_mul(T(2), f[1])), f[3]), f[4]), rn_mul(T(2), f[6])), rn_mul(T(2), f[7])), rn_mul(T(2), f[9])), rn_mul(T(4), f[12])), rn_mul(T(2), f[13])), rn_mul(T(2), f[17])), rn_mul(T(4), f[22])), rn_mul(T(4), f[26]));
  rho = rn_div(scmf, s);
}
template <typename T>
PSL_HDI void mirror_n25(T (&f)[27]) {
  f[2] = f[1];
  f[5] = f[6];
  f[8] = f[9];
  f[10] = f[7];
  f[11] = f[12];
  f[14] = f[17];
  f[15] = f[12];
  f[16] = f[12];
  f[18] = f[13];
  f[19] = f[22];
  f[20] = f[26];
  f[21] = f[26];
  f[23] = f[22];
  f[24] = f[26];
  f[25] = f[22];
}

// ---- outer normal (+0,-1,-1): 15 unknown populations ----
template <typename T>
PSL_HDI void mbbc_n9(T (&f)[27], const T rho, const T ux, const T uy, const T uz) {
  const T smf0 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(f[0], f[1]), f[2]), f[3]), f[5]), f[7]), f[10]), f[11]), f[16]), f[18]), f[23]), f[25]);
  const T smf1 = rn_sub(rn_add(rn_add(rn_sub(rn_sub(rn_add(rn_sub(f[1], f[2]), f[7]), f[10]), f[11]), f[16]), f[23]), f[25]);
  const T smf2 = rn_sub(rn_sub(rn_sub(rn_sub(rn_sub((-f[5]), f[11]), f[16]), f[18]), f[23]), f[25]);
  const T smf3 = rn_sub(rn_sub(rn_sub(rn_sub(rn_sub((-f[3]), f[7]), f[10]), f[18]), f[23]), f[25]);
  const T smf4 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(f[1], f[2]), f[7]), f[10]), f[11]), f[16]), f[23]), f[25]);
  const T smf5 = rn_add(rn_add(rn_add(rn_add(rn_add(f[5], f[11]), f[16]), f[18]), f[23]), f[25]);
  const T smf6 = rn_add(rn_add(rn_add(rn_add(rn_add(f[3], f[7]), f[10]), f[18]), f[23]), f[25]);
  const T smf7 = rn_add(rn_sub(rn_add((-f[7]), f[10]), f[23]), f[25]);
  const T smf8 = rn_add(rn_sub(rn_sub(f[11], f[16]), f[23]), f[25]);
  const T smf9 = rn_sub(rn_sub(rn_sub((-f[11]), f[16]), f[23]), f[25]);
  const T smf10 = rn_sub(rn_sub(rn_sub((-f[7]), f[10]), f[23]), f[25]);
  const T smf11 = rn_sub(rn_add(rn_add((-f[11]), f[16]), f[23]), f[25]);
  const T smf12 = rn_sub(rn_add(rn_sub(f[7], f[10]), f[23]), f[25]);
  const T smf13 = rn_add(rn_add(rn_add(f[7], f[10]), f[23]), f[25]);
  const T smf14 = rn_add(rn_add(rn_add(f[11], f[16]), f[23]), f[25]);
  const T m0 = rho;
  const T m1 = rn_mul(rho, ux);
  const T m2 = rn_mul(rho, uy);
  const T m3 = rn_mul(rho, uz);
  const T m4 = rn_add(rn_mul((T(1) / T(3)), rho), rn_mul(rn_mul(rho, ux), ux));
  const T m5 = rn_add(rn_mul((T(1) / T(3)), rho), rn_mul(rn_mul(rho, uy), uy));
  const T m6 = rn_add(rn_mul((T(1) / T(3)), rho), rn_mul(rn_mul(rho, uz), uz));
  const T m7 = rn_mul(rn_mul(rho, ux), uz);
  const T m8 = rn_mul(rn_mul(rho, ux), uy);
  const T m9 = rn_add(rn_mul(rn_mul((T(1) / T(3)), rho), uy), rn_mul(rn_mul(rn_mul(rho, ux), ux), uy));
  const T m10 = rn_add(rn_mul(rn_mul((T(1) / T(3)), rho), uz), rn_mul(rn_mul(rn_mul(rho, ux), ux), uz));
  const T m11 = rn_add(rn_mul(rn_mul((T(1) / T(3)), rho), ux), rn_mul(rn_mul(rn_mul(rho, ux), uy), uy));
  const T m12 = rn_add(rn_mul(rn_mul((T(1) / T(3)), rho), ux), rn_mul(rn_mul(rn_mul(rho, ux), uz), uz));
  const T m13 = rn_add(rn_add(rn_add(rn_mul((T(1) / T(9)), rho), rn_mul(rn_mul(rn_mul((T(1) / T(3)), rho), ux), ux)), rn_mul(rn_mul(rn_mul((T(1) / T(3)), rho), uz), uz)), rn_mul(rn_mul(rn_mul(rn_mul(rho, ux), ux), uz), uz));
  const T m14 = rn_add(rn_add(rn_add(rn_mul((T(1) / T(9)), rho), rn_mul(rn_mul(rn_mul((T(1) / T(3)), rho), ux), ux)), rn_mul(rn_mul(rn_mul((T(1) / T(3)), rho), uy), uy)), rn_mul(rn_mul(rn_mul(rn_mul(rho, ux), ux), uy), uy));
  const T s0 = rn_sub(m0, smf0);
  const T s1 = rn_sub(m1, smf1);
  const T s2 = rn_sub(m2, smf2);
  const T s3 = rn_sub(m3, smf3);
  const T s4 = rn_sub(m4, smf4);
  const T s5 = rn_sub(m5, smf5);
  const T s6 = rn_sub(m6, smf6);
  const T s7 = rn_sub(m7, smf7);
  const T s8 = rn_sub(m8, smf8);
  const T s9 = rn_sub(m9, smf9);
  const T s10 = rn_sub(m10, smf10);
  const T s11 = rn_sub(m11, smf11);
  const T s12 = rn_sub(m12, smf12);
  const T s13 = rn_sub(m13, smf13);
  const T s14 = rn_sub(m14, smf14);
  f[4] = rn_add(rn_sub(rn_sub(s0, s4), s5), s14);
  f[6] = rn_add(rn_sub(rn_sub(s0, s4), s6), s13);
  f[8] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(2)), s1), rn_mul((T(1) / T(2)), s4)), rn_mul((T(1) / T(2)), s11)), rn_mul((T(-1) / T(2)), s14));
  f[9] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), s1), rn_mul((T(1) / T(2)), s4)), rn_mul((T(-1) / T(2)), s11)), rn_mul((T(-1) / T(2)), s14));
  f[12] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), s1), rn_mul((T(1) / T(2)), s4)), rn_mul((T(-1) / T(2)), s12)), rn_mul((T(-1) / T(2)), s13));
  f[13] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(2)), s3), rn_mul((T(1) / T(2)), s6)), rn_mul((T(1) / T(2)), s10)), rn_mul((T(-1) / T(2)), s13));
  f[14] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(2)), s2), rn_mul((T(1) / T(2)), s5)), rn_mul((T(1) / T(2)), s9)), rn_mul((T(-1) / T(2)), s14));
  f[15] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(2)), s1), rn_mul((T(1) / T(2)), s4)), rn_mul((T(1) / T(2)), s12)), rn_mul((T(-1) / T(2)), s13));
  f[17] = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add((-s0), rn_mul((T(1) / T(2)), s2)), rn_mul((T(1) / T(2)), s3)), s4), rn_mul((T(1) / T(2)), s5)), rn_mul((T(1) / T(2)), s6)), rn_mul((T(-1) / T(2)), s9)), rn_mul((T(-1) / T(2)), s10)), rn_mul((T(-1) / T(2)), s13)), rn_mul((T(-1) / T(2)), s14));
  f[19] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(4)), s7), rn_mul((T(-1) / T(4)), s10)), rn_mul((T(-1) / T(4)), s12)), rn_mul((T(1) / T(4)), s13));
  f[20] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(4)), s8), rn_mul((T(-1) / T(4)), s9)), rn_mul((T(1) / T(4)), s11)), rn_mul((T(1) / T(4)), s14));
  f[21] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(4)), s8), rn_mul((T(-1) / T(4)), s9)), rn_mul((T(-1) / T(4)), s11)), rn_mul((T(1) / T(4)), s14));
  f[22] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(4)), s7), rn_mul((T(-1) / T(4)), s10)), rn_mul((T(1) / T(4)), s12)), rn_mul((T(1) / T(4)), s13));
  f[24] = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), s1), rn_mul((T(-1) / T(2)), s4)), rn_mul((T(-1) / T(4)), s7)), rn_mul((T(-1) / T(4)), s8)), rn_mul((T(1) / T(4)), s9)), rn_mul((T(1) / T(4)), s10)), rn_mul((T(-1) / T(4)), s11)), rn_mul((T(-1) / T(4)), s12)), rn_mul((T(1) / T(4)), s13)), rn_mul((T(1) / T(4)), s14));
  f[26] = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_mul((T(-1) / T(2)), s1), rn_mul((T(-1) / T(2)), s4)), rn_mul((T(1) / T(4)), s7)), rn_mul((T(1) / T(4)), s8)), rn_mul((T(1) / T(4)), s9)), rn_mul((T(1) / T(4)), s10)), rn_mul((T(1) / T(4)), s11)), rn_mul((T(1) / T(4)), s12)), rn_mul((T(1) / T(4)), s13)), rn_mul((T(1) / T(4)), s14));
}
template <typename T>
PSL_HDI void restore_rho_u_n9(const T (&f)[27], T& rho, T& ux, T& uy, T& uz) {
  const T q0 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_mul(T(2), f[0]), rn_mul(T(2), f[1])), rn_mul(T(2), f[2])), f[3]), f[5]), f[7]), f[10]), f[11]), f[16]), rn_mul(T(-4), f[18])), rn_mul(T(-4), f[23])), rn_mul(T(-4), f[25]));
  const T q1 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_sub(f[1], f[2]), rn_mul(T(2), f[7])), rn_mul(T(-2), f[10])), rn_mul(T(-2), f[11])), rn_mul(T(2), f[16])), rn_mul(T(4), f[23])), rn_mul(T(-4), f[25]));
  const T q2 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), f[0]), rn_mul((T(1) / T(2)), f[1])), rn_mul((T(1) / T(2)), f[2])), f[3]), rn_mul(T(-2), f[5])), f[7]), f[10]), rn_mul(T(-2), f[11])), rn_mul(T(-2), f[16])), rn_mul(T(-4), f[18])), rn_mul(T(-4), f[23])), rn_mul(T(-4), f[25]));
  const T q3 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), f[0]), rn_mul((T(1) / T(2)), f[1])), rn_mul((T(1) / T(2)), f[2])), rn_mul(T(-2), f[3])), f[5]), rn_mul(T(-2), f[7])), rn_mul(T(-2), f[10])), f[11]), f[16]), rn_mul(T(-4), f[18])), rn_mul(T(-4), f[23])), rn_mul(T(-4), f[25]));
  rho = q0;
  ux = rn_div(q1, rho);
  uy = rn_div(q2, rho);
  uz = rn_div(q3, rho);
}
template <typename T>
PSL_HDI void restore_u_n9(const T (&f)[27], const T rho, T& ux, T& uy, T& uz) {
  const T scmf0 = rn_div(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(f[0], f[1]), f[2]), rn_mul(T(2), f[3])), rn_mul(T(2), f[5])), rn_mul(T(2), f[7])), rn_mul(T(2), f[10])), rn_mul(T(2), f[11])), rn_mul(T(2), f[16])), rn_mul(T(4), f[18])), rn_mul(T(4), f[23])), rn_mul(T(4), f[25])), rho);
  const T scmf1 = rn_div(rn_add(rn_add(rn_add(rn_add(rn_add(f[0], f[1]), f[2]), rn_mul(T(2), f[3])), rn_mul(T(2), f[7])), rn_mul(T(2), f[10])), rho);
  const T scmf2 = rn_div(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_sub(f[1], f[2]), rn_mul(T(2), f[7])), rn_mul(T(-2), f[10])), rn_mul(T(-2), f[11])), rn_mul(T(2), f[16])), rn_mul(T(4), f[23])), rn_mul(T(-4), f[25])), rho);
  const T s0 = rn_sub(scmf0, T(1));
  const T s1 = rn_sub(scmf1, (T(2) / T(3)));
  const T s2 = rn_sub(scmf2, T(0));
  ux = s2;
  uy = rn_add((-s0), rn_mul((T(3) / T(2)), s1));
  uz = rn_mul((T(-3) / T(2)), s1);
}
template <typename T>
PSL_HDI void restore_rho_n9(const T (&f)[27], T& rho, const T ux, const T uy, const T uz) {
  const T scqu = rn_add(rn_mul(T(-1), uy), rn_mul(T(-1), uz));
  const T s = rn_add(T(1), scqu);
  const T scmf = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(f[0], f[1]), f[2]), rn_mul(T(2), f[3])), rn_mul(T(2), f[5])), rn_mul(T(2), f[7])), rn_mul(T(2), f[10])), rn_mul(T(2), f[11])), rn_mul(T(2), f[16])), rn_mul(T(4), f[18])), rn_mul(T(4), f[23])), rn_mul(T(4), f[25]));
  rho = rn_div(scmf, s);
}
template <typename T>
PSL_HDI void mirror_n9(T (&f)[27]) {
  f[4] = f[3];
  f[6] = f[5];
  f[8] = f[10];
  f[9] = f[7];
  f[12] = f[16];
  f[13] = f[18];
  f[14] = f[18];
  f[15] = f[11];
  f[17] = f[18];
  f[19] = f[25];
  f[20] = f[23];
  f[21] = f[25];
  f[22] = f[23];
  f[24] = f[25];
  f[26] = f[23];
}

// ---- outer normal (-1,+0,-1): 15 unknown populations ----
template <typename T>
PSL_HDI void mbbc_n3(T (&f)[27], const T rho, const T ux, const T uy, const T uz) {
  const T smf0 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(f[0], f[2]), f[3]), f[5]), f[6]), f[10]), f[11]), f[13]), f[15]), f[18]), f[19]), f[25]);
  const T smf1 = rn_sub(rn_sub(rn_sub(rn_sub(rn_sub((-f[2]), f[10]), f[11]), f[15]), f[19]), f[25]);
  const T smf2 = rn_sub(rn_add(rn_sub(rn_add(rn_add(rn_sub(rn_add((-f[5]), f[6]), f[11]), f[13]), f[15]), f[18]), f[19]), f[25]);
  const T smf3 = rn_sub(rn_sub(rn_sub(rn_sub(rn_sub((-f[3]), f[10]), f[13]), f[18]), f[19]), f[25]);
  const T smf4 = rn_add(rn_add(rn_add(rn_add(rn_add(f[2], f[10]), f[11]), f[15]), f[19]), f[25]);
  const T smf5 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(f[5], f[6]), f[11]), f[13]), f[15]), f[18]), f[19]), f[25]);
  const T smf6 = rn_add(rn_add(rn_add(rn_add(rn_add(f[3], f[10]), f[13]), f[18]), f[19]), f[25]);
  const T smf7 = rn_add(rn_sub(rn_add((-f[13]), f[18]), f[19]), f[25]);
  const T smf8 = rn_add(rn_sub(rn_sub(f[11], f[15]), f[19]), f[25]);
  const T smf9 = rn_sub(rn_add(rn_add((-f[11]), f[15]), f[19]), f[25]);
  const T smf10 = rn_sub(rn_sub(rn_sub((-f[11]), f[15]), f[19]), f[25]);
  const T smf11 = rn_sub(rn_sub(rn_sub((-f[13]), f[18]), f[19]), f[25]);
  const T smf12 = rn_sub(rn_add(rn_sub(f[13], f[18]), f[19]), f[25]);
  const T smf13 = rn_add(rn_add(rn_add(f[13], f[18]), f[19]), f[25]);
  const T smf14 = rn_add(rn_add(rn_add(f[11], f[15]), f[19]), f[25]);
  const T m0 = rho;
  const T m1 = rn_mul(rho, ux);
  const T m2 = rn_mul(rho, uy);
  const T m3 = rn_mul(rho, uz);
  const T m4 = rn_add(rn_mul((T(1) / T(3)), rho), rn_mul(rn_mul(rho, ux), ux));
  const T m5 = rn_add(rn_mul((T(1) / T(3)), rho), rn_mul(rn_mul(rho, uy), uy));
  const T m6 = rn_add(rn_mul((T(1) / T(3)), rho), rn_mul(rn_mul(rho, uz), uz));
  const T m7 = rn_mul(rn_mul(rho, uy), uz);
  const T m8 = rn_mul(rn_mul(rho, ux), uy);
  const T m9 = rn_add(rn_mul(rn_mul((T(1) / T(3)), rho), uy), rn_mul(rn_mul(rn_mul(rho, ux), ux), uy));
  const T m10 = rn_add(rn_mul(rn_mul((T(1) / T(3)), rho), ux), rn_mul(rn_mul(rn_mul(rho, ux), uy), uy));
  const T m11 = rn_add(rn_mul(rn_mul((T(1) / T(3)), rho), uz), rn_mul(rn_mul(rn_mul(rho, uy), uy), uz));
  const T m12 = rn_add(rn_mul(rn_mul((T(1) / T(3)), rho), uy), rn_mul(rn_mul(rn_mul(rho, uy), uz), uz));
  const T m13 = rn_add(rn_add(rn_add(rn_mul((T(1) / T(9)), rho), rn_mul(rn_mul(rn_mul((T(1) / T(3)), rho), uy), uy)), rn_mul(rn_mul(rn_mul((T(1) / T(3)), rho), uz), uz)), rn_mul(rn_mul(rn_mul(rn_mul(rho, uy), uy), uz), uz));
  const T m14 = rn_add(rn_add(rn_add(rn_mul((T(1) / T(9)), rho), rn_mul(rn_mul(rn_mul((T(1) / T(3)), rho), ux), ux)), rn_mul(rn_mul(rn_mul((T(1) / T(3)), rho), uy), uy)), rn_mul(rn_mul(rn_mul(rn_mul(rho, ux), ux), uy), uy));
  const T s0 = rn_sub(m0, smf0);
  const T s1 = rn_sub(m1, smf1);
  const T s2 = rn_sub(m2, smf2);
  const T s3 = rn_sub(m3, smf3);
  const T s4 = rn_sub(m4, smf4);
  const T s5 = rn_sub(m5, smf5);
  const T s6 = rn_sub(m6, smf6);
  const T s7 = rn_sub(m7, smf7);
  const T s8 = rn_sub(m8, smf8);
  const T s9 = rn_sub(m9, smf9);
  const T s10 = rn_sub(m10, smf10);
  const T s11 = rn_sub(m11, smf11);
  const T s12 = rn_sub(m12, smf12);
  const T s13 = rn_sub(m13, smf13);
  const T s14 = rn_sub(m14, smf14);
  f[1] = rn_add(rn_sub(rn_sub(s0, s5), s6), s13);
  f[4] = rn_add(rn_sub(rn_sub(s0, s4), s5), s14);
  f[7] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(2)), s3), rn_mul((T(1) / T(2)), s6)), rn_mul((T(1) / T(2)), s11)), rn_mul((T(-1) / T(2)), s13));
  f[8] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(2)), s1), rn_mul((T(1) / T(2)), s4)), rn_mul((T(1) / T(2)), s10)), rn_mul((T(-1) / T(2)), s14));
  f[9] = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add((-s0), rn_mul((T(1) / T(2)), s1)), rn_mul((T(1) / T(2)), s3)), rn_mul((T(1) / T(2)), s4)), s5), rn_mul((T(1) / T(2)), s6)), rn_mul((T(-1) / T(2)), s10)), rn_mul((T(-1) / T(2)), s11)), rn_mul((T(-1) / T(2)), s13)), rn_mul((T(-1) / T(2)), s14));
  f[12] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), s2), rn_mul((T(1) / T(2)), s5)), rn_mul((T(-1) / T(2)), s12)), rn_mul((T(-1) / T(2)), s13));
  f[14] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(2)), s2), rn_mul((T(1) / T(2)), s5)), rn_mul((T(1) / T(2)), s9)), rn_mul((T(-1) / T(2)), s14));
  f[16] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(2)), s2), rn_mul((T(1) / T(2)), s5)), rn_mul((T(1) / T(2)), s12)), rn_mul((T(-1) / T(2)), s13));
  f[17] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), s2), rn_mul((T(1) / T(2)), s5)), rn_mul((T(-1) / T(2)), s9)), rn_mul((T(-1) / T(2)), s14));
  f[20] = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), s2), rn_mul((T(-1) / T(2)), s5)), rn_mul((T(-1) / T(4)), s7)), rn_mul((T(-1) / T(4)), s8)), rn_mul((T(-1) / T(4)), s9)), rn_mul((T(1) / T(4)), s10)), rn_mul((T(1) / T(4)), s11)), rn_mul((T(-1) / T(4)), s12)), rn_mul((T(1) / T(4)), s13)), rn_mul((T(1) / T(4)), s14));
  f[21] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(4)), s8), rn_mul((T(-1) / T(4)), s9)), rn_mul((T(-1) / T(4)), s10)), rn_mul((T(1) / T(4)), s14));
  f[22] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(4)), s7), rn_mul((T(-1) / T(4)), s11)), rn_mul((T(1) / T(4)), s12)), rn_mul((T(1) / T(4)), s13));
  f[23] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(4)), s7), rn_mul((T(-1) / T(4)), s11)), rn_mul((T(-1) / T(4)), s12)), rn_mul((T(1) / T(4)), s13));
  f[24] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(4)), s8), rn_mul((T(1) / T(4)), s9)), rn_mul((T(-1) / T(4)), s10)), rn_mul((T(1) / T(4)), s14));
  f[26] = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_mul((T(-1) / T(2)), s2), rn_mul((T(-1) / T(2)), s5)), rn_mul((T(1) / T(4)), s7)), rn_mul((T(1) / T(4)), s8)), rn_mul((T(1) / T(4)), s9)), rn_mul((T(1) / T(4)), s10)), rn_mul((T(1) / T(4)), s11)), rn_mul((T(1) / T(4)), s12)), rn_mul((T(1) / T(4)), s13)), rn_mul((T(1) / T(4)), s14));
}
template <typename T>
PSL_HDI void restore_rho_u_n3(const T (&f)[27], T& rho, T& ux, T& uy, T& uz) {
  const T q0 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_mul(T(2), f[0]), f[2]), f[3]), rn_mul(T(2), f[5])), rn_mul(T(2), f[6])), rn_mul(T(-4), f[10])), f[11]), f[13]), f[15]), f[18]), rn_mul(T(-4), f[19])), rn_mul(T(-4), f[25]));
  const T q1 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), f[0]), rn_mul(T(-2), f[2])), f[3]), rn_mul((T(1) / T(2)), f[5])), rn_mul((T(1) / T(2)), f[6])), rn_mul(T(-4), f[10])), rn_mul(T(-2), f[11])), f[13]), rn_mul(T(-2), f[15])), f[18]), rn_mul(T(-4), f[19])), rn_mul(T(-4), f[25]));
  const T q2 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add((-f[5]), f[6]), rn_mul(T(-2), f[11])), rn_mul(T(2), f[13])), rn_mul(T(2), f[15])), rn_mul(T(-2), f[18])), rn_mul(T(4), f[19])), rn_mul(T(-4), f[25]));
  const T q3 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), f[0]), f[2]), rn_mul(T(-2), f[3])), rn_mul((T(1) / T(2)), f[5])), rn_mul((T(1) / T(2)), f[6])), rn_mul(T(-4), f[10])), f[11]), rn_mul(T(-2), f[13])), f[15]), rn_mul(T(-2), f[18])), rn_mul(T(-4), f[19])), rn_mul(T(-4), f[25]));
  rho = q0;
  ux = rn_div(q1, rho);
  uy = rn_div(q2, rho);
  uz = rn_div(q3, rho);
}
template <typename T>
PSL_HDI void restore_u_n3(const T (&f)[27], const T rho, T& ux, T& uy, T& uz) {
  const T scmf0 = rn_div(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(f[0], rn_mul(T(2), f[2])), rn_mul(T(2), f[3])), f[5]), f[6]), rn_mul(T(4), f[10])), rn_mul(T(2), f[11])), rn_mul(T(2), f[13])), rn_mul(T(2), f[15])), rn_mul(T(2), f[18])), rn_mul(T(4), f[19])), rn_mul(T(4), f[25])), rho);
  const T scmf1 = rn_div(rn_add(rn_add(rn_add(rn_add(rn_add(f[0], rn_mul(T(2), f[3])), f[5]), f[6]), rn_mul(T(2), f[13])), rn_mul(T(2), f[18])), rho);
  const T scmf2 = rn_div(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add((-f[5]), f[6]), rn_mul(T(-2), f[11])), rn_mul(T(2), f[13])), rn_mul(T(2), f[15])), rn_mul(T(-2), f[18])), rn_mul(T(4), f[19])), rn_mul(T(-4), f[25])), rho);
  const T s0 = rn_sub(scmf0, T(1));
  const T s1 = rn_sub(scmf1, (T(2) / T(3)));
  const T s2 = rn_sub(scmf2, T(0));
  ux = rn_add((-s0), rn_mul((T(3) / T(2)), s1));
  uy = s2;
  uz = rn_mul((T(-3) / T(2)), s1);
}
template <typename T>
PSL_HDI void restore_rho_n3(const T (&f)[27], T& rho, const T ux, const T uy, const T uz) {
  const T scqu = rn_add(rn_mul(T(-1), ux), rn_mul(T(-1), uz));
  const T s = rn_add(T(1), scqu);
  const T scmf = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(f[0], rn_mul(T(2), f[2])), rn_mul(T(2), f[3])), f[5]), f[6]), rn_mul(T(4), f[10])), rn_mul(T(2), f[11])), rn_mul(T(2), f[13])), rn_mul(T(2), f[15])), rn_mul(T(2), f[18])), rn_mul(T(4), f[19])), rn_mul(T(4), f[25]));
  rho = rn_div(scmf, s);
}
template <typename T>
PSL_HDI void mirror_n3(T (&f)[27]) {
  f[1] = f[2];
  f[4] = f[3];
  f[7] = f[10];
  f[8] = f[10];
  f[9] = f[10];
  f[12] = f[15];
  f[14] = f[18];
  f[16] = f[11];
  f[17] = f[13];
  f[20] = f[25];
  f[21] = f[25];
  f[22] = f[19];
  f[23] = f[25];
  f[24] = f[19];
  f[26] = f[19];
}

// ---- outer normal (-1,-1,+0): 15 unknown populations ----
template <typename T>
PSL_HDI void mbbc_n1(T (&f)[27], const T rho, const T ux, const T uy, const T uz) {
  const T smf0 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(f[0], f[2]), f[3]), f[4]), f[5]), f[8]), f[10]), f[11]), f[14]), f[18]), f[21]), f[25]);
  const T smf1 = rn_sub(rn_sub(rn_sub(rn_sub(rn_sub((-f[2]), f[8]), f[10]), f[11]), f[21]), f[25]);
  const T smf2 = rn_sub(rn_sub(rn_sub(rn_sub(rn_sub((-f[5]), f[11]), f[14]), f[18]), f[21]), f[25]);
  const T smf3 = rn_sub(rn_add(rn_sub(rn_add(rn_sub(rn_add(rn_add((-f[3]), f[4]), f[8]), f[10]), f[14]), f[18]), f[21]), f[25]);
  const T smf4 = rn_add(rn_add(rn_add(rn_add(rn_add(f[2], f[8]), f[10]), f[11]), f[21]), f[25]);
  const T smf5 = rn_add(rn_add(rn_add(rn_add(rn_add(f[5], f[11]), f[14]), f[18]), f[21]), f[25]);
  const T smf6 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(f[3], f[4]), f[8]), f[10]), f[14]), f[18]), f[21]), f[25]);
  const T smf7 = rn_add(rn_sub(rn_add((-f[14]), f[18]), f[21]), f[25]);
  const T smf8 = rn_add(rn_sub(rn_add((-f[8]), f[10]), f[21]), f[25]);
  const T smf9 = rn_sub(rn_add(rn_sub(f[8], f[10]), f[21]), f[25]);
  const T smf10 = rn_sub(rn_add(rn_sub(f[14], f[18]), f[21]), f[25]);
  const T smf11 = rn_sub(rn_sub(rn_sub((-f[8]), f[10]), f[21]), f[25]);
  const T smf12 = rn_sub(rn_sub(rn_sub((-f[14]), f[18]), f[21]), f[25]);
  const T smf13 = rn_add(rn_add(rn_add(f[14], f[18]), f[21]), f[25]);
  const T smf14 = rn_add(rn_add(rn_add(f[8], f[10]), f[21]), f[25]);
  const T m0 = rho;
  const T m1 = rn_mul(rho, ux);
  const T m2 = rn_mul(rho, uy);
  const T m3 = rn_mul(rho, uz);
  const T m4 = rn_add(rn_mul((T(1) / T(3)), rho), rn_mul(rn_mul(rho, ux), ux));
  const T m5 = rn_add(rn_mul((T(1) / T(3)), rho), rn_mul(rn_mul(rho, uy), uy));
  const T m6 = rn_add(rn_mul((T(1) / T(3)), rho), rn_mul(rn_mul(rho, uz), uz));
  const T m7 = rn_mul(rn_mul(rho, uy), uz);
  const T m8 = rn_mul(rn_mul(rho, ux), uz);
  const T m9 = rn_add(rn_mul(rn_mul((T(1) / T(3)), rho), uz), rn_mul(rn_mul(rn_mul(rho, ux), ux), uz));
  const T m10 = rn_add(rn_mul(rn_mul((T(1) / T(3)), rho), uz), rn_mul(rn_mul(rn_mul(rho, uy), uy), uz));
  const T m11 = rn_add(rn_mul(rn_mul((T(1) / T(3)), rho), ux), rn_mul(rn_mul(rn_mul(rho, ux), uz), uz));
  const T m12 = rn_add(rn_mul(rn_mul((T(1) / T(3)), rho), uy), rn_mul(rn_mul(rn_mul(rho, uy), uz), uz));
  const T m13 = rn_add(rn_add(rn_add(rn_mul((T(1) / T(9)), rho), rn_mul(rn_mul(rn_mul((T(1) / T(3)), rho), uy), uy)), rn_mul(rn_mul(rn_mul((T(1) / T(3)), rho), uz), uz)), rn_mul(rn_mul(rn_mul(rn_mul(rho, uy), uy), uz), uz));
  const T m14 = rn_add(rn_add(rn_add(rn_mul((T(1) / T(9)), rho), rn_mul(rn_mul(rn_mul((T(1) / T(3)), rho), ux), ux)), rn_mul(rn_mul(rn_mul((T(1) / T(3)), rho), uz), uz)), rn_mul(rn_mul(rn_mul(rn_mul(rho, ux), ux), uz), uz));
  const T s0 = rn_sub(m0, smf0);
  const T s1 = rn_sub(m1, smf1);
  const T s2 = rn_sub(m2, smf2);
  const T s3 = rn_sub(m3, smf3);
  const T s4 = rn_sub(m4, smf4);
  const T s5 = rn_sub(m5, smf5);
  const T s6 = rn_sub(m6, smf6);
  const T s7 = rn_sub(m7, smf7);
  const T s8 = rn_sub(m8, smf8);
  const T s9 = rn_sub(m9, smf9);
  const T s10 = rn_sub(m10, smf10);
  const T s11 = rn_sub(m11, smf11);
  const T s12 = rn_sub(m12, smf12);
  const T s13 = rn_sub(m13, smf13);
  const T s14 = rn_sub(m14, smf14);
  f[1] = rn_add(rn_sub(rn_sub(s0, s5), s6), s13);
  f[6] = rn_add(rn_sub(rn_sub(s0, s4), s6), s14);
  f[7] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(2)), s3), rn_mul((T(1) / T(2)), s6)), rn_mul((T(1) / T(2)), s10)), rn_mul((T(-1) / T(2)), s13));
  f[9] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), s3), rn_mul((T(1) / T(2)), s6)), rn_mul((T(-1) / T(2)), s10)), rn_mul((T(-1) / T(2)), s13));
  f[12] = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add((-s0), rn_mul((T(1) / T(2)), s1)), rn_mul((T(1) / T(2)), s2)), rn_mul((T(1) / T(2)), s4)), rn_mul((T(1) / T(2)), s5)), s6), rn_mul((T(-1) / T(2)), s11)), rn_mul((T(-1) / T(2)), s12)), rn_mul((T(-1) / T(2)), s13)), rn_mul((T(-1) / T(2)), s14));
  f[13] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(2)), s3), rn_mul((T(1) / T(2)), s6)), rn_mul((T(1) / T(2)), s9)), rn_mul((T(-1) / T(2)), s14));
  f[15] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(2)), s1), rn_mul((T(1) / T(2)), s4)), rn_mul((T(1) / T(2)), s11)), rn_mul((T(-1) / T(2)), s14));
  f[16] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(2)), s2), rn_mul((T(1) / T(2)), s5)), rn_mul((T(1) / T(2)), s12)), rn_mul((T(-1) / T(2)), s13));
  f[17] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), s3), rn_mul((T(1) / T(2)), s6)), rn_mul((T(-1) / T(2)), s9)), rn_mul((T(-1) / T(2)), s14));
  f[19] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(4)), s8), rn_mul((T(-1) / T(4)), s9)), rn_mul((T(-1) / T(4)), s11)), rn_mul((T(1) / T(4)), s14));
  f[20] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(4)), s7), rn_mul((T(1) / T(4)), s10)), rn_mul((T(-1) / T(4)), s12)), rn_mul((T(1) / T(4)), s13));
  f[22] = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), s3), rn_mul((T(-1) / T(2)), s6)), rn_mul((T(-1) / T(4)), s7)), rn_mul((T(-1) / T(4)), s8)), rn_mul((T(-1) / T(4)), s9)), rn_mul((T(-1) / T(4)), s10)), rn_mul((T(1) / T(4)), s11)), rn_mul((T(1) / T(4)), s12)), rn_mul((T(1) / T(4)), s13)), rn_mul((T(1) / T(4)), s14));
  f[23] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(4)), s7), rn_mul((T(-1) / T(4)), s10)), rn_mul((T(-1) / T(4)), s12)), rn_mul((T(1) / T(4)), s13));
  f[24] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(4)), s8), rn_mul((T(1) / T(4)), s9)), rn_mul((T(-1) / T(4)), s11)), rn_mul((T(1) / T(4)), s14));
  f[26] = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_mul((T(-1) / T(2)), s3), rn_mul((T(-1) / T(2)), s6)), rn_mul((T(1) / T(4)), s7)), rn_mul((T(1) / T(4)), s8)), rn_mul((T(1) / T(4)), s9)), rn_mul((T(1) / T(4)), s10)), rn_mul((T(1) / T(4)), s11)), rn_mul((T(1) / T(4)), s12)), rn_mul((T(1) / T(4)), s13)), rn_mul((T(1) / T(4)), s14));
}
template <typename T>
PSL_HDI void restore_rho_u_n1(const T (&f)[27], T& rho, T& ux, T& uy, T& uz) {
  const T q0 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_mul(T(2), f[0]), f[2]), rn_mul(T(2), f[3])), rn_mul(T(2), f[4])), f[5]), f[8]), f[10]), rn_mul(T(-4), f[11])), f[14]), f[18]), rn_mul(T(-4), f[21])), rn_mul(T(-4), f[25]));
  const T q1 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), f[0]), rn_mul(T(-2), f[2])), rn_mul((T(1) / T(2)), f[3])), rn_mul((T(1) / T(2)), f[4])), f[5]), rn_mul(T(-2), f[8])), rn_mul(T(-2), f[10])), rn_mul(T(-4), f[11])), f[14]), f[18]), rn_mul(T(-4), f[21])), rn_mul(T(-4), f[25]));
  const T q2 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), f[0]), f[2]), rn_mul((T(1) / T(2)), f[3])), rn_mul((T(1) / T(2)), f[4])), rn_mul(T(-2), f[5])), f[8]), f[10]), rn_mul(T(-4), f[11])), rn_mul(T(-2), f[14])), rn_mul(T(-2), f[18])), rn_mul(T(-4), f[21])), rn_mul(T(-4), f[25]));
  const T q3 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add((-f[3]), f[4]), rn_mul(T(2), f[8])), rn_mul(T(-2), f[10])), rn_mul(T(2), f[14])), rn_mul(T(-2), f[18])), rn_mul(T(4), f[21])), rn_mul(T(-4), f[25]));
  rho = q0;
  ux = rn_div(q1, rho);
  uy = rn_div(q2, rho);
  uz = rn_div(q3, rho);
}
template <typename T>
PSL_HDI void restore_u_n1(const T (&f)[27], const T rho, T& ux, T& uy, T& uz) {
  const T scmf0 = rn_div(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(f[0], rn_mul(T(2), f[2])), f[3]), f[4]), rn_mul(T(2), f[5])), rn_mul(T(2), f[8])), rn_mul(T(2), f[10])), rn_mul(T(4), f[11])), rn_mul(T(2), f[14])), rn_mul(T(2), f[18])), rn_mul(T(4), f[21])), rn_mul(T(4), f[25])), rho);
  const T scmf1 = rn_div(rn_add(rn_add(rn_add(rn_add(rn_add(f[0], f[3]), f[4]), rn_mul(T(2), f[5])), rn_mul(T(2), f[14])), rn_mul(T(2), f[18])), rho);
  const T scmf2 = rn_div(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add((-f[3]), f[4]), rn_mul(T(2), f[8])), rn_mul(T(-2), f[10])), rn_mul(T(2), f[14])), rn_mul(T(-2), f[18])), rn_mul(T(4), f[21])), rn_mul(T(-4), f[25])), rho);
  const T s0 = rn_sub(scmf0, T(1));
  const T s1 = rn_sub(scmf1, (T(2) / T(3)));
  const T s2 = rn_sub(scmf2, T(0));
  ux = rn_add((-s0), rn_mul((T(3) / T(2)), s1));
  uy = rn_mul((T(-3) / T(2)), s1);
  uz = s2;
}
template <typename T>
PSL_HDI void restore_rho_n1(const T (&f)[27], T& rho, const T ux, const T uy, const T uz) {
  const T scqu = rn_add(rn_mul(T(-1), ux), rn_mul(T(-1), uy));
  const T s = rn_add(T(1), scqu);
  const T scmf = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(f[0], rn_mul(T(2), f[2])), f[3]), f[4]), rn_mul(T(2), f[5])), rn_mul(T(2), f[8])), rn_mul(T(2), f[10])), rn_mul(T(4), f[11])), rn_mul(T(2), f[14])), rn_mul(T(2), f[18])), rn_mul(T(4), f[21])), rn_mul(T(4), f[25]));
  rho = rn_div(scmf, s);
}
template <typename T>
PSL_HDI void mirror_n1(T (&f)[27]) {
  f[1] = f[2];
  f[6] = f[5];
  f[7] = f[10];
  f[9] = f[8];
  f[12] = f[11];
  f[13] = f[18];
  f[15] = f[11];
  f[16] = f[11];
  f[17] = f[14];
  f[19] = f[25];
  f[20] = f[21];
  f[22] = f[25];
  f[23] = f[25];
  f[24] = f[21];
  f[26] = f[21];
}

// ---- outer normal (+0,+1,-1): 15 unknown populations ----
template <typename T>
PSL_HDI void mbbc_n15(T (&f)[27], const T rho, const T ux, const T uy, const T uz) {
  const T smf0 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(f[0], f[1]), f[2]), f[3]), f[6]), f[7]), f[10]), f[12]), f[13]), f[15]), f[19]), f[22]);
  const T smf1 = rn_add(rn_sub(rn_sub(rn_add(rn_sub(rn_add(rn_sub(f[1], f[2]), f[7]), f[10]), f[12]), f[15]), f[19]), f[22]);
  const T smf2 = rn_add(rn_add(rn_add(rn_add(rn_add(f[6], f[12]), f[13]), f[15]), f[19]), f[22]);
  const T smf3 = rn_sub(rn_sub(rn_sub(rn_sub(rn_sub((-f[3]), f[7]), f[10]), f[13]), f[19]), f[22]);
  const T smf4 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(f[1], f[2]), f[7]), f[10]), f[12]), f[15]), f[19]), f[22]);
  const T smf5 = rn_add(rn_add(rn_add(rn_add(rn_add(f[6], f[12]), f[13]), f[15]), f[19]), f[22]);
  const T smf6 = rn_add(rn_add(rn_add(rn_add(rn_add(f[3], f[7]), f[10]), f[13]), f[19]), f[22]);
  const T smf7 = rn_sub(rn_add(rn_add((-f[7]), f[10]), f[19]), f[22]);
  const T smf8 = rn_add(rn_sub(rn_sub(f[12], f[15]), f[19]), f[22]);
  const T smf9 = rn_add(rn_add(rn_add(f[12], f[15]), f[19]), f[22]);
  const T smf10 = rn_sub(rn_sub(rn_sub((-f[7]), f[10]), f[19]), f[22]);
  const T smf11 = rn_add(rn_sub(rn_sub(f[12], f[15]), f[19]), f[22]);
  const T smf12 = rn_add(rn_sub(rn_sub(f[7], f[10]), f[19]), f[22]);
  const T smf13 = rn_add(rn_add(rn_add(f[7], f[10]), f[19]), f[22]);
  const T smf14 = rn_add(rn_add(rn_add(f[12], f[15]), f[19]), f[22]);
  const T m0 = rho;
  const T m1 = rn_mul(rho, ux);
  const T m2 = rn_mul(rho, uy);
  const T m3 = rn_mul(rho, uz);
  const T m4 = rn_add(rn_mul((T(1) / T(3)), rho), rn_mul(rn_mul(rho, ux), ux));
  const T m5 = rn_add(rn_mul((T(1) / T(3)), rho), rn_mul(rn_mul(rho, uy), uy));
  const T m6 = rn_add(rn_mul((T(1) / T(3)), rho), rn_mul(rn_mul(rho, uz), uz));
  const T m7 = rn_mul(rn_mul(rho, ux), uz);
  const T m8 = rn_mul(rn_mul(rho, ux), uy);
  const T m9 = rn_add(rn_mul(rn_mul((T(1) / T(3)), rho), uy), rn_mul(rn_mul(rn_mul(rho, ux), ux), uy));
  const T m10 = rn_add(rn_mul(rn_mul((T(1) / T(3)), rho), uz), rn_mul(rn_mul(rn_mul(rho, ux), ux), uz));
  const T m11 = rn_add(rn_mul(rn_mul((T(1) / T(3)), rho), ux), rn_mul(rn_mul(rn_mul(rho, ux), uy), uy));
  const T m12 = rn_add(rn_mul(rn_mul((T(1) / T(3)), rho), ux), rn_mul(rn_mul(rn_mul(rho, ux), uz), uz));
  const T m13 = rn_add(rn_add(rn_add(rn_mul((T(1) / T(9)), rho), rn_mul(rn_mul(rn_mul((T(1) / T(3)), rho), ux), ux)), rn_mul(rn_mul(rn_mul((T(1) / T(3)), rho), uz), uz)), rn_mul(rn_mul(rn_mul(rn_mul(rho, ux), ux), uz), uz));
  const T m14 = rn_add(rn_add(rn_add(rn_mul((T(1) / T(9)), rho), rn_mul(rn_mul(rn_mul((T(1) / T(3)), rho), ux), ux)), rn_mul(rn_mul(rn_mul((T(1) / T(3)), rho), uy), uy)), rn_mul(rn_mul(rn_mul(rn_mul(rho, ux), ux), uy), uy));
  const T s0 = rn_sub(m0, smf0);
  const T s1 = rn_sub(m1, smf1);
  const T s2 = rn_sub(m2, smf2);
  const T s3 = rn_sub(m3, smf3);
  const T s4 = rn_sub(m4, smf4);
  const T s5 = rn_sub(m5, smf5);
  const T s6 = rn_sub(m6, smf6);
  const T s7 = rn_sub(m7, smf7);
  const T s8 = rn_sub(m8, smf8);
  const T s9 = rn_sub(m9, smf9);
  const T s10 = rn_sub(m10, smf10);
  const T s11 = rn_sub(m11, smf11);
  const T s12 = rn_sub(m12, smf12);
  const T s13 = rn_sub(m13, smf13);
  const T s14 = rn_sub(m14, smf14);
  f[4] = rn_add(rn_sub(rn_sub(s0, s4), s5), s14);
  f[5] = rn_add(rn_sub(rn_sub(s0, s4), s6), s13);
  f[8] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(2)), s1), rn_mul((T(1) / T(2)), s4)), rn_mul((T(1) / T(2)), s11)), rn_mul((T(-1) / T(2)), s14));
  f[9] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), s1), rn_mul((T(1) / T(2)), s4)), rn_mul((T(-1) / T(2)), s11)), rn_mul((T(-1) / T(2)), s14));
  f[11] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(2)), s1), rn_mul((T(1) / T(2)), s4)), rn_mul((T(1) / T(2)), s12)), rn_mul((T(-1) / T(2)), s13));
  f[14] = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add((-s0), rn_mul((T(-1) / T(2)), s2)), rn_mul((T(1) / T(2)), s3)), s4), rn_mul((T(1) / T(2)), s5)), rn_mul((T(1) / T(2)), s6)), rn_mul((T(1) / T(2)), s9)), rn_mul((T(-1) / T(2)), s10)), rn_mul((T(-1) / T(2)), s13)), rn_mul((T(-1) / T(2)), s14));
  f[16] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), s1), rn_mul((T(1) / T(2)), s4)), rn_mul((T(-1) / T(2)), s12)), rn_mul((T(-1) / T(2)), s13));
  f[17] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), s2), rn_mul((T(1) / T(2)), s5)), rn_mul((T(-1) / T(2)), s9)), rn_mul((T(-1) / T(2)), s14));
  f[18] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(2)), s3), rn_mul((T(1) / T(2)), s6)), rn_mul((T(1) / T(2)), s10)), rn_mul((T(-1) / T(2)), s13));
  f[20] = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_mul((T(-1) / T(2)), s1), rn_mul((T(-1) / T(2)), s4)), rn_mul((T(1) / T(4)), s7)), rn_mul((T(-1) / T(4)), s8)), rn_mul((T(-1) / T(4)), s9)), rn_mul((T(1) / T(4)), s10)), rn_mul((T(1) / T(4)), s11)), rn_mul((T(1) / T(4)), s12)), rn_mul((T(1) / T(4)), s13)), rn_mul((T(1) / T(4)), s14));
  f[21] = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), s1), rn_mul((T(-1) / T(2)), s4)), rn_mul((T(-1) / T(4)), s7)), rn_mul((T(1) / T(4)), s8)), rn_mul((T(-1) / T(4)), s9)), rn_mul((T(1) / T(4)), s10)), rn_mul((T(-1) / T(4)), s11)), rn_mul((T(-1) / T(4)), s12)), rn_mul((T(1) / T(4)), s13)), rn_mul((T(1) / T(4)), s14));
  f[23] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(4)), s7), rn_mul((T(-1) / T(4)), s10)), rn_mul((T(1) / T(4)), s12)), rn_mul((T(1) / T(4)), s13));
  f[24] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(4)), s8), rn_mul((T(1) / T(4)), s9)), rn_mul((T(-1) / T(4)), s11)), rn_mul((T(1) / T(4)), s14));
  f[25] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(4)), s7), rn_mul((T(-1) / T(4)), s10)), rn_mul((T(-1) / T(4)), s12)), rn_mul((T(1) / T(4)), s13));
  f[26] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(4)), s8), rn_mul((T(1) / T(4)), s9)), rn_mul((T(1) / T(4)), s11)), rn_mul((T(1) / T(4)), s14));
}
template <typename T>
PSL_HDI void restore_rho_u_n15(const T (&f)[27], T& rho, T& ux, T& uy, T& uz) {
  const T q0 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_mul(T(2), f[0]), rn_mul(T(2), f[1])), rn_mul(T(2), f[2])), f[3]), f[6]), f[7]), f[10]), f[12]), rn_mul(T(-4), f[13])), f[15]), rn_mul(T(-4), f[19])), rn_mul(T(-4), f[22]));
  const T q1 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_sub(f[1], f[2]), rn_mul(T(2), f[7])), rn_mul(T(-2), f[10])), rn_mul(T(2), f[12])), rn_mul(T(-2), f[15])), rn_mul(T(-4), f[19])), rn_mul(T(4), f[22]));
  const T q2 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_sub(rn_sub(rn_add(rn_sub(rn_add(rn_add(rn_mul((T(-1) / T(2)), f[0]), rn_mul((T(-1) / T(2)), f[1])), rn_mul((T(-1) / T(2)), f[2])), f[3]), rn_mul(T(2), f[6])), f[7]), f[10]), rn_mul(T(2), f[12])), rn_mul(T(4), f[13])), rn_mul(T(2), f[15])), rn_mul(T(4), f[19])), rn_mul(T(4), f[22]));
  const T q3 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), f[0]), rn_mul((T(1) / T(2)), f[1])), rn_mul((T(1) / T(2)), f[2])), rn_mul(T(-2), f[3])), f[6]), rn_mul(T(-2), f[7])), rn_mul(T(-2), f[10])), f[12]), rn_mul(T(-4), f[13])), f[15]), rn_mul(T(-4), f[19])), rn_mul(T(-4), f[22]));
  rho = q0;
  ux = rn_div(q1, rho);
  uy = rn_div(q2, rho);
  uz = rn_div(q3, rho);
}
template <typename T>
PSL_HDI void restore_u_n15(const T (&f)[27], const T rho, T& ux, T& uy, T& uz) {
  const T scmf0 = rn_div(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_sub(rn_sub((-f[0]), f[1]), f[2]), rn_mul(T(-2), f[3])), rn_mul(T(-2), f[6])), rn_mul(T(-2), f[7])), rn_mul(T(-2), f[10])), rn_mul(T(-2), f[12])), rn_mul(T(-4), f[13])), rn_mul(T(-2), f[15])), rn_mul(T(-4), f[19])), rn_mul(T(-4), f[22])), rho);
  const T scmf1 = rn_div(rn_add(rn_add(rn_add(rn_add(rn_add(f[0], f[1]), f[2]), rn_mul(T(2), f[3])), rn_mul(T(2), f[7])), rn_mul(T(2), f[10])), rho);
  const T scmf2 = rn_div(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add((-f[1]), f[2]), rn_mul(T(-2), f[7])), rn_mul(T(2), f[10])), rn_mul(T(-2), f[12])), rn_mul(T(2), f[15])), rn_mul(T(4), f[19])), rn_mul(T(-4), f[22])), rho);
  const T s0 = rn_sub(scmf0, T(-1));
  const T s1 = rn_sub(scmf1, (T(2) / T(3)));
  const T s2 = rn_sub(scmf2, T(0));
  ux = (-s2);
  uy = rn_add((-s0), rn_mul((T(-3) / T(2)), s1));
  uz = rn_mul((T(-3) / T(2)), s1);
}
template <typename T>
PSL_HDI void restore_rho_n15(const T (&f)[27], T& rho, const T ux, const T uy, const T uz) {
  const T scqu = rn_add(rn_mul(T(-1), uy), rn_mul(T(1), uz));
  const T s = rn_add(T(-1), scqu);
  const T scmf = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_sub(rn_sub((-f[0]), f[1]), f[2]), rn_mul(T(-2), f[3])), rn_mul(T(-2), f[6])), rn_mul(T(-2), f[7])), rn_mul(T(-2), f[10])), rn_mul(T(-2), f[12])), rn_mul(T(-4), f[13])), rn_mul(T(-2), f[15])), rn_mul(T(-4), f[19])), rn_mul(T(-4), f[22]));
  rho = rn_div(scmf, s);
}
template <typename T>
PSL_HDI void mirror_n15(T (&f)[27]) {
  f[4] = f[3];
  f[5] = f[6];
  f[8] = f[10];
  f[9] = f[7];
  f[11] = f[15];
  f[14] = f[13];
  f[16] = f[12];
  f[17] = f[13];
  f[18] = f[13];
  f[20] = f[22];
  f[21] = f[19];
  f[23] = f[22];
  f[24] = f[19];
  f[25] = f[19];
  f[26] = f[22];
}

// ---- outer normal (+1,+0,-1): 15 unknown populations ----
template <typename T>
PSL_HDI void mbbc_n21(T (&f)[27], const T rho, const T ux, const T uy, const T uz) {
  const T smf0 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(f[0], f[1]), f[3]), f[5]), f[6]), f[7]), f[12]), f[13]), f[16]), f[18]), f[22]), f[23]);
  const T smf1 = rn_add(rn_add(rn_add(rn_add(rn_add(f[1], f[7]), f[12]), f[16]), f[22]), f[23]);
  const T smf2 = rn_sub(rn_add(rn_sub(rn_sub(rn_add(rn_add(rn_add((-f[5]), f[6]), f[12]), f[13]), f[16]), f[18]), f[22]), f[23]);
  const T smf3 = rn_sub(rn_sub(rn_sub(rn_sub(rn_sub((-f[3]), f[7]), f[13]), f[18]), f[22]), f[23]);
  const T smf4 = rn_add(rn_add(rn_add(rn_add(rn_add(f[1], f[7]), f[12]), f[16]), f[22]), f[23]);
  const T smf5 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(f[5], f[6]), f[12]), f[13]), f[16]), f[18]), f[22]), f[23]);
  const T smf6 = rn_add(rn_add(rn_add(rn_add(rn_add(f[3], f[7]), f[13]), f[18]), f[22]), f[23]);
  const T smf7 = rn_add(rn_sub(rn_add((-f[13]), f[18]), f[22]), f[23]);
  const T smf8 = rn_sub(rn_add(rn_sub(f[12], f[16]), f[22]), f[23]);
  const T smf9 = rn_sub(rn_add(rn_sub(f[12], f[16]), f[22]), f[23]);
  const T smf10 = rn_add(rn_add(rn_add(f[12], f[16]), f[22]), f[23]);
  const T smf11 = rn_sub(rn_sub(rn_sub((-f[13]), f[18]), f[22]), f[23]);
  const T smf12 = rn_sub(rn_add(rn_sub(f[13], f[18]), f[22]), f[23]);
  const T smf13 = rn_add(rn_add(rn_add(f[13], f[18]), f[22]), f[23]);
  const T smf14 = rn_add(rn_add(rn_add(f[12], f[16]), f[22]), f[23]);
  const T m0 = rho;
  const T m1 = rn_mul(rho, ux);
  const T m2 = rn_mul(rho, uy);
  const T m3 = rn_mul(rho, uz);
  const T m4 = rn_add(rn_mul((T(1) / T(3)), rho), rn_mul(rn_mul(rho, ux), ux));
  const T m5 = rn_add(rn_mul((T(1) / T(3)), rho), rn_mul(rn_mul(rho, uy), uy));
  const T m6 = rn_add(rn_mul((T(1) / T(3)), rho), rn_mul(rn_mul(rho, uz), uz));
  const T m7 = rn_mul(rn_mul(rho, uy), uz);
  const T m8 = rn_mul(rn_mul(rho, ux), uy);
  const T m9 = rn_add(rn_mul(rn_mul((T(1) / T(3)), rho), uy), rn_mul(rn_mul(rn_mul(rho, ux), ux), uy));
  const T m10 = rn_add(rn_mul(rn_mul((T(1) / T(3)), rho), ux), rn_mul(rn_mul(rn_mul(rho, ux), uy), uy));
  const T m11 = rn_add(rn_mul(rn_mul((T(1) / T(3)), rho), uz), rn_mul(rn_mul(rn_mul(rho, uy), uy), uz));
  const T m12 = rn_add(rn_mul(rn_mul((T(1) / T(3)), rho), uy), rn_mul(rn_mul(rn_mul(rho, uy), uz), uz));
  const T m13 = rn_add(rn_add(rn_add(rn_mul((T(1) / T(9)), rho), rn_mul(rn_mul(rn_mul((T(1) / T(3)), rho), uy), uy)), rn_mul(rn_mul(rn_mul((T(1) / T(3)), rho), uz), uz)), rn_mul(rn_mul(rn_mul(rn_mul(rho, uy), uy), uz), uz));
  const T m14 = rn_add(rn_add(rn_add(rn_mul((T(1) / T(9)), rho), rn_mul(rn_mul(rn_mul((T(1) / T(3)), rho), ux), ux)), rn_mul(rn_mul(rn_mul((T(1) / T(3)), rho), uy), uy)), rn_mul(rn_mul(rn_mul(rn_mul(rho, ux), ux), uy), uy));
  const T s0 = rn_sub(m0, smf0);
  const T s1 = rn_sub(m1, smf1);
  const T s2 = rn_sub(m2, smf2);
  const T s3 = rn_sub(m3, smf3);
  const T s4 = rn_sub(m4, smf4);
  const T s5 = rn_sub(m5, smf5);
  const T s6 = rn_sub(m6, smf6);
  const T s7 = rn_sub(m7, smf7);
  const T s8 = rn_sub(m8, smf8);
  const T s9 = rn_sub(m9, smf9);
  const T s10 = rn_sub(m10, smf10);
  const T s11 = rn_sub(m11, smf11);
  const T s12 = rn_sub(m12, smf12);
  const T s13 = rn_sub(m13, smf13);
  const T s14 = rn_sub(m14, smf14);
  f[2] = rn_add(rn_sub(rn_sub(s0, s5), s6), s13);
  f[4] = rn_add(rn_sub(rn_sub(s0, s4), s5), s14);
  f[8] = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add((-s0), rn_mul((T(-1) / T(2)), s1)), rn_mul((T(1) / T(2)), s3)), rn_mul((T(1) / T(2)), s4)), s5), rn_mul((T(1) / T(2)), s6)), rn_mul((T(1) / T(2)), s10)), rn_mul((T(-1) / T(2)), s11)), rn_mul((T(-1) / T(2)), s13)), rn_mul((T(-1) / T(2)), s14));
  f[9] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), s1), rn_mul((T(1) / T(2)), s4)), rn_mul((T(-1) / T(2)), s10)), rn_mul((T(-1) / T(2)), s14));
  f[10] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(2)), s3), rn_mul((T(1) / T(2)), s6)), rn_mul((T(1) / T(2)), s11)), rn_mul((T(-1) / T(2)), s13));
  f[11] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(2)), s2), rn_mul((T(1) / T(2)), s5)), rn_mul((T(1) / T(2)), s12)), rn_mul((T(-1) / T(2)), s13));
  f[14] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(2)), s2), rn_mul((T(1) / T(2)), s5)), rn_mul((T(1) / T(2)), s9)), rn_mul((T(-1) / T(2)), s14));
  f[15] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), s2), rn_mul((T(1) / T(2)), s5)), rn_mul((T(-1) / T(2)), s12)), rn_mul((T(-1) / T(2)), s13));
  f[17] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), s2), rn_mul((T(1) / T(2)), s5)), rn_mul((T(-1) / T(2)), s9)), rn_mul((T(-1) / T(2)), s14));
  f[19] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(4)), s7), rn_mul((T(-1) / T(4)), s11)), rn_mul((T(1) / T(4)), s12)), rn_mul((T(1) / T(4)), s13));
  f[20] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(4)), s8), rn_mul((T(-1) / T(4)), s9)), rn_mul((T(1) / T(4)), s10)), rn_mul((T(1) / T(4)), s14));
  f[21] = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), s2), rn_mul((T(-1) / T(2)), s5)), rn_mul((T(-1) / T(4)), s7)), rn_mul((T(1) / T(4)), s8)), rn_mul((T(-1) / T(4)), s9)), rn_mul((T(-1) / T(4)), s10)), rn_mul((T(1) / T(4)), s11)), rn_mul((T(-1) / T(4)), s12)), rn_mul((T(1) / T(4)), s13)), rn_mul((T(1) / T(4)), s14));
  f[24] = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_mul((T(-1) / T(2)), s2), rn_mul((T(-1) / T(2)), s5)), rn_mul((T(1) / T(4)), s7)), rn_mul((T(-1) / T(4)), s8)), rn_mul((T(1) / T(4)), s9)), rn_mul((T(-1) / T(4)), s10)), rn_mul((T(1) / T(4)), s11)), rn_mul((T(1) / T(4)), s12)), rn_mul((T(1) / T(4)), s13)), rn_mul((T(1) / T(4)), s14));
  f[25] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(4)), s7), rn_mul((T(-1) / T(4)), s11)), rn_mul((T(-1) / T(4)), s12)), rn_mul((T(1) / T(4)), s13));
  f[26] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(4)), s8), rn_mul((T(1) / T(4)), s9)), rn_mul((T(1) / T(4)), s10)), rn_mul((T(1) / T(4)), s14));
}
template <typename T>
PSL_HDI void restore_rho_u_n21(const T (&f)[27], T& rho, T& ux, T& uy, T& uz) {
  const T q0 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_mul(T(2), f[0]), f[1]), f[3]), rn_mul(T(2), f[5])), rn_mul(T(2), f[6])), rn_mul(T(-4), f[7])), f[12]), f[13]), f[16]), f[18]), rn_mul(T(-4), f[22])), rn_mul(T(-4), f[23]));
  const T q1 = rn_add(rn_add(rn_sub(rn_add(rn_sub(rn_add(rn_add(rn_add(rn_add(rn_sub(rn_add(rn_mul((T(-1) / T(2)), f[0]), rn_mul(T(2), f[1])), f[3]), rn_mul((T(-1) / T(2)), f[5])), rn_mul((T(-1) / T(2)), f[6])), rn_mul(T(4), f[7])), rn_mul(T(2), f[12])), f[13]), rn_mul(T(2), f[16])), f[18]), rn_mul(T(4), f[22])), rn_mul(T(4), f[23]));
  const T q2 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add((-f[5]), f[6]), rn_mul(T(2), f[12])), rn_mul(T(2), f[13])), rn_mul(T(-2), f[16])), rn_mul(T(-2), f[18])), rn_mul(T(4), f[22])), rn_mul(T(-4), f[23]));
  const T q3 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), f[0]), f[1]), rn_mul(T(-2), f[3])), rn_mul((T(1) / T(2)), f[5])), rn_mul((T(1) / T(2)), f[6])), rn_mul(T(-4), f[7])), f[12]), rn_mul(T(-2), f[13])), f[16]), rn_mul(T(-2), f[18])), rn_mul(T(-4), f[22])), rn_mul(T(-4), f[23]));
  rho = q0;
  ux = rn_div(q1, rho);
  uy = rn_div(q2, rho);
  uz = rn_div(q3, rho);
}
template <typename T>
PSL_HDI void restore_u_n21(const T (&f)[27], const T rho, T& ux, T& uy, T& uz) {
  const T scmf0 = rn_div(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_sub(rn_sub(rn_add(rn_add((-f[0]), rn_mul(T(-2), f[1])), rn_mul(T(-2), f[3])), f[5]), f[6]), rn_mul(T(-4), f[7])), rn_mul(T(-2), f[12])), rn_mul(T(-2), f[13])), rn_mul(T(-2), f[16])), rn_mul(T(-2), f[18])), rn_mul(T(-4), f[22])), rn_mul(T(-4), f[23])), rho);
  const T scmf1 = rn_div(rn_add(rn_add(rn_add(rn_add(rn_add(f[0], rn_mul(T(2), f[3])), f[5]), f[6]), rn_mul(T(2), f[13])), rn_mul(T(2), f[18])), rho);
  const T scmf2 = rn_div(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_sub(f[5], f[6]), rn_mul(T(-2), f[12])), rn_mul(T(-2), f[13])), rn_mul(T(2), f[16])), rn_mul(T(2), f[18])), rn_mul(T(-4), f[22])), rn_mul(T(4), f[23])), rho);
  const T s0 = rn_sub(scmf0, T(-1));
  const T s1 = rn_sub(scmf1, (T(2) / T(3)));
  const T s2 = rn_sub(scmf2, T(0));
  ux = rn_add((-s0), rn_mul((T(-3) / T(2)), s1));
  uy = (-s2);
  uz = rn_mul((T(-3) / T(2)), s1);
}
template <typename T>
PSL_HDI void restore_rho_n21(const T (&f)[27], T& rho, const T ux, const T uy, const T uz) {
  const T scqu = rn_add(rn_mul(T(-1), ux), rn_mul(T(1), uz));
  const T s = rn_add(T(-1), scqu);
  const T scmf = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_sub(rn_sub(rn_add(rn_add((-f[0]), rn_mul(T(-2), f[1])), rn_mul(T(-2), f[3])), f[5]), f[6]), rn_mul(T(-4), f[7])), rn_mul(T(-2), f[12])), rn_mul(T(-2), f[13])), rn_mul(T(-2), f[16])), rn_mul(T(-2), f[18])), rn_mul(T(-4), f[22])), rn_mul(T(-4), f[23]));
  rho = rn_div(scmf, s);
}
template <typename T>
PSL_HDI void mirror_n21(T (&f)[27]) {
  f[2] = f[1];
  f[4] = f[3];
  f[8] = f[7];
  f[9] = f[7];
  f[10] = f[7];
  f[11] = f[16];
  f[14] = f[18];
  f[15] = f[12];
  f[17] = f[13];
  f[19] = f[22];
  f[20] = f[23];
  f[21] = f[23];
  f[24] = f[22];
  f[25] = f[23];
  f[26] = f[22];
}

// ---- outer normal (+1,-1,+0): 15 unknown populations ----
template <typename T>
PSL_HDI void mbbc_n19(T (&f)[27], const T rho, const T ux, const T uy, const T uz) {
  const T smf0 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(f[0], f[1]), f[3]), f[4]), f[5]), f[7]), f[9]), f[14]), f[16]), f[18]), f[20]), f[23]);
  const T smf1 = rn_add(rn_add(rn_add(rn_add(rn_add(f[1], f[7]), f[9]), f[16]), f[20]), f[23]);
  const T smf2 = rn_sub(rn_sub(rn_sub(rn_sub(rn_sub((-f[5]), f[14]), f[16]), f[18]), f[20]), f[23]);
  const T smf3 = rn_sub(rn_add(rn_sub(rn_add(rn_add(rn_sub(rn_add((-f[3]), f[4]), f[7]), f[9]), f[14]), f[18]), f[20]), f[23]);
  const T smf4 = rn_add(rn_add(rn_add(rn_add(rn_add(f[1], f[7]), f[9]), f[16]), f[20]), f[23]);
  const T smf5 = rn_add(rn_add(rn_add(rn_add(rn_add(f[5], f[14]), f[16]), f[18]), f[20]), f[23]);
  const T smf6 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(f[3], f[4]), f[7]), f[9]), f[14]), f[18]), f[20]), f[23]);
  const T smf7 = rn_add(rn_sub(rn_add((-f[14]), f[18]), f[20]), f[23]);
  const T smf8 = rn_sub(rn_add(rn_add((-f[7]), f[9]), f[20]), f[23]);
  const T smf9 = rn_sub(rn_add(rn_add((-f[7]), f[9]), f[20]), f[23]);
  const T smf10 = rn_sub(rn_add(rn_sub(f[14], f[18]), f[20]), f[23]);
  const T smf11 = rn_add(rn_add(rn_add(f[7], f[9]), f[20]), f[23]);
  const T smf12 = rn_sub(rn_sub(rn_sub((-f[14]), f[18]), f[20]), f[23]);
  const T smf13 = rn_add(rn_add(rn_add(f[14], f[18]), f[20]), f[23]);
  const T smf14 = rn_add(rn_add(rn_add(f[7], f[9]), f[20]), f[23]);
  const T m0 = rho;
  const T m1 = rn_mul(rho, ux);
  const T m2 = rn_mul(rho, uy);
  const T m3 = rn_mul(rho, uz);
  const T m4 = rn_add(rn_mul((T(1) / T(3)), rho), rn_mul(rn_mul(rho, ux), ux));
  const T m5 = rn_add(rn_mul((T(1) / T(3)), rho), rn_mul(rn_mul(rho, uy), uy));
  const T m6 = rn_add(rn_mul((T(1) / T(3)), rho), rn_mul(rn_mul(rho, uz), uz));
  const T m7 = rn_mul(rn_mul(rho, uy), uz);
  const T m8 = rn_mul(rn_mul(rho, ux), uz);
  const T m9 = rn_add(rn_mul(rn_mul((T(1) / T(3)), rho), uz), rn_mul(rn_mul(rn_mul(rho, ux), ux), uz));
  const T m10 = rn_add(rn_mul(rn_mul((T(1) / T(3)), rho), uz), rn_mul(rn_mul(rn_mul(rho, uy), uy), uz));
  const T m11 = rn_add(rn_mul(rn_mul((T(1) / T(3)), rho), ux), rn_mul(rn_mul(rn_mul(rho, ux), uz), uz));
  const T m12 = rn_add(rn_mul(rn_mul((T(1) / T(3)), rho), uy), rn_mul(rn_mul(rn_mul(rho, uy), uz), uz));
  const T m13 = rn_add(rn_add(rn_add(rn_mul((T(1) / T(9)), rho), rn_mul(rn_mul(rn_mul((T(1) / T(3)), rho), uy), uy)), rn_mul(rn_mul(rn_mul((T(1) / T(3)), rho), uz), uz)), rn_mul(rn_mul(rn_mul(rn_mul(rho, uy), uy), uz), uz));
  const T m14 = rn_add(rn_add(rn_add(rn_mul((T(1) / T(9)), rho), rn_mul(rn_mul(rn_mul((T(1) / T(3)), rho), ux), ux)), rn_mul(rn_mul(rn_mul((T(1) / T(3)), rho), uz), uz)), rn_mul(rn_mul(rn_mul(rn_mul(rho, ux), ux), uz), uz));
  const T s0 = rn_sub(m0, smf0);
  const T s1 = rn_sub(m1, smf1);
  const T s2 = rn_sub(m2, smf2);
  const T s3 = rn_sub(m3, smf3);
  const T s4 = rn_sub(m4, smf4);
  const T s5 = rn_sub(m5, smf5);
  const T s6 = rn_sub(m6, smf6);
  const T s7 = rn_sub(m7, smf7);
  const T s8 = rn_sub(m8, smf8);
  const T s9 = rn_sub(m9, smf9);
  const T s10 = rn_sub(m10, smf10);
  const T s11 = rn_sub(m11, smf11);
  const T s12 = rn_sub(m12, smf12);
  const T s13 = rn_sub(m13, smf13);
  const T s14 = rn_sub(m14, smf14);
  f[2] = rn_add(rn_sub(rn_sub(s0, s5), s6), s13);
  f[6] = rn_add(rn_sub(rn_sub(s0, s4), s6), s14);
  f[8] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), s3), rn_mul((T(1) / T(2)), s6)), rn_mul((T(-1) / T(2)), s10)), rn_mul((T(-1) / T(2)), s13));
  f[10] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(2)), s3), rn_mul((T(1) / T(2)), s6)), rn_mul((T(1) / T(2)), s10)), rn_mul((T(-1) / T(2)), s13));
  f[11] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(2)), s2), rn_mul((T(1) / T(2)), s5)), rn_mul((T(1) / T(2)), s12)), rn_mul((T(-1) / T(2)), s13));
  f[12] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), s1), rn_mul((T(1) / T(2)), s4)), rn_mul((T(-1) / T(2)), s11)), rn_mul((T(-1) / T(2)), s14));
  f[13] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(2)), s3), rn_mul((T(1) / T(2)), s6)), rn_mul((T(1) / T(2)), s9)), rn_mul((T(-1) / T(2)), s14));
  f[15] = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add((-s0), rn_mul((T(-1) / T(2)), s1)), rn_mul((T(1) / T(2)), s2)), rn_mul((T(1) / T(2)), s4)), rn_mul((T(1) / T(2)), s5)), s6), rn_mul((T(1) / T(2)), s11)), rn_mul((T(-1) / T(2)), s12)), rn_mul((T(-1) / T(2)), s13)), rn_mul((T(-1) / T(2)), s14));
  f[17] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), s3), rn_mul((T(1) / T(2)), s6)), rn_mul((T(-1) / T(2)), s9)), rn_mul((T(-1) / T(2)), s14));
  f[19] = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), s3), rn_mul((T(-1) / T(2)), s6)), rn_mul((T(-1) / T(4)), s7)), rn_mul((T(1) / T(4)), s8)), rn_mul((T(-1) / T(4)), s9)), rn_mul((T(-1) / T(4)), s10)), rn_mul((T(-1) / T(4)), s11)), rn_mul((T(1) / T(4)), s12)), rn_mul((T(1) / T(4)), s13)), rn_mul((T(1) / T(4)), s14));
  f[21] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(4)), s7), rn_mul((T(1) / T(4)), s10)), rn_mul((T(-1) / T(4)), s12)), rn_mul((T(1) / T(4)), s13));
  f[22] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(4)), s8), rn_mul((T(-1) / T(4)), s9)), rn_mul((T(1) / T(4)), s11)), rn_mul((T(1) / T(4)), s14));
  f[24] = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_mul((T(-1) / T(2)), s3), rn_mul((T(-1) / T(2)), s6)), rn_mul((T(1) / T(4)), s7)), rn_mul((T(-1) / T(4)), s8)), rn_mul((T(1) / T(4)), s9)), rn_mul((T(1) / T(4)), s10)), rn_mul((T(-1) / T(4)), s11)), rn_mul((T(1) / T(4)), s12)), rn_mul((T(1) / T(4)), s13)), rn_mul((T(1) / T(4)), s14));
  f[25] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(4)), s7), rn_mul((T(-1) / T(4)), s10)), rn_mul((T(-1) / T(4)), s12)), rn_mul((T(1) / T(4)), s13));
  f[26] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(4)), s8), rn_mul((T(1) / T(4)), s9)), rn_mul((T(1) / T(4)), s11)), rn_mul((T(1) / T(4)), s14));
}
template <typename T>
PSL_HDI void restore_rho_u_n19(const T (&f)[27], T& rho, T& ux, T& uy, T& uz) {
  const T q0 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_mul(T(2), f[0]), f[1]), rn_mul(T(2), f[3])), rn_mul(T(2), f[4])), f[5]), f[7]), f[9]), f[14]), rn_mul(T(-4), f[16])), f[18]), rn_mul(T(-4), f[20])), rn_mul(T(-4), f[23]));
  const T q1 = rn_add(rn_add(rn_sub(rn_add(rn_sub(rn_add(rn_add(rn_sub(rn_add(rn_add(rn_add(rn_mul((T(-1) / T(2)), f[0]), rn_mul(T(2), f[1])), rn_mul((T(-1) / T(2)), f[3])), rn_mul((T(-1) / T(2)), f[4])), f[5]), rn_mul(T(2), f[7])), rn_mul(T(2), f[9])), f[14]), rn_mul(T(4), f[16])), f[18]), rn_mul(T(4), f[20])), rn_mul(T(4), f[23]));
  const T q2 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), f[0]), f[1]), rn_mul((T(1) / T(2)), f[3])), rn_mul((T(1) / T(2)), f[4])), rn_mul(T(-2), f[5])), f[7]), f[9]), rn_mul(T(-2), f[14])), rn_mul(T(-4), f[16])), rn_mul(T(-2), f[18])), rn_mul(T(-4), f[20])), rn_mul(T(-4), f[23]));
  const T q3 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add((-f[3]), f[4]), rn_mul(T(-2), f[7])), rn_mul(T(2), f[9])), rn_mul(T(2), f[14])), rn_mul(T(-2), f[18])), rn_mul(T(4), f[20])), rn_mul(T(-4), f[23]));
  rho = q0;
  ux = rn_div(q1, rho);
  uy = rn_div(q2, rho);
  uz = rn_div(q3, rho);
}
template <typename T>
PSL_HDI void restore_u_n19(const T (&f)[27], const T rho, T& ux, T& uy, T& uz) {
  const T scmf0 = rn_div(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_sub(rn_sub(rn_add((-f[0]), rn_mul(T(-2), f[1])), f[3]), f[4]), rn_mul(T(-2), f[5])), rn_mul(T(-2), f[7])), rn_mul(T(-2), f[9])), rn_mul(T(-2), f[14])), rn_mul(T(-4), f[16])), rn_mul(T(-2), f[18])), rn_mul(T(-4), f[20])), rn_mul(T(-4), f[23])), rho);
  const T scmf1 = rn_div(rn_add(rn_add(rn_add(rn_add(rn_add(f[0], f[3]), f[4]), rn_mul(T(2), f[5])), rn_mul(T(2), f[14])), rn_mul(T(2), f[18])), rho);
  const T scmf2 = rn_div(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_sub(f[3], f[4]), rn_mul(T(2), f[7])), rn_mul(T(-2), f[9])), rn_mul(T(-2), f[14])), rn_mul(T(2), f[18])), rn_mul(T(-4), f[20])), rn_mul(T(4), f[23])), rho);
  const T s0 = rn_sub(scmf0, T(-1));
  const T s1 = rn_sub(scmf1, (T(2) / T(3)));
  const T s2 = rn_sub(scmf2, T(0));
  ux = rn_add((-s0), rn_mul((T(-3) / T(2)), s1));
  uy = rn_mul((T(-3) / T(2)), s1);
  uz = (-s2);
}
template <typename T>
PSL_HDI void restore_rho_n19(const T (&f)[27], T& rho, const T ux, const T uy, const T uz) {
  const T scqu = rn_add(rn_mul(T(-1), ux), rn_mul(T(1), uy));
  const T s = rn_add(T(-1), scqu);
  const T scmf = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_sub(rn_sub(rn_add((-f[0]), rn_mul(T(-2), f[1])), f[3]), f[4]), rn_mul(T(-2), f[5])), rn_mul(T(-2), f[7])), rn_mul(T(-2), f[9])), rn_mul(T(-2), f[14])), rn_mul(T(-4), f[16])), rn_mul(T(-2), f[18])), rn_mul(T(-4), f[20])), rn_mul(T(-4), f[23]));
  rho = rn_div(scmf, s);
}
template <typename T>
PSL_HDI void mirror_n19(T (&f)[27]) {
  f[2] = f[1];
  f[6] = f[5];
  f[8] = f[9];
  f[10] = f[7];
  f[11] = f[16];
  f[12] = f[16];
  f[13] = f[18];
  f[15] = f[16];
  f[17] = f[14];
  f[19] = f[23];
  f[21] = f[20];
  f[22] = f[23];
  f[24] = f[20];
  f[25] = f[23];
  f[26] = f[20];
}

// ---- outer normal (+0,-1,+1): 15 unknown populations ----
template <typename T>
PSL_HDI void mbbc_n11(T (&f)[27], const T rho, const T ux, const T uy, const T uz) {
  const T smf0 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(f[0], f[1]), f[2]), f[4]), f[5]), f[8]), f[9]), f[11]), f[14]), f[16]), f[20]), f[21]);
  const T smf1 = rn_sub(rn_add(rn_add(rn_sub(rn_add(rn_sub(rn_sub(f[1], f[2]), f[8]), f[9]), f[11]), f[16]), f[20]), f[21]);
  const T smf2 = rn_sub(rn_sub(rn_sub(rn_sub(rn_sub((-f[5]), f[11]), f[14]), f[16]), f[20]), f[21]);
  const T smf3 = rn_add(rn_add(rn_add(rn_add(rn_add(f[4], f[8]), f[9]), f[14]), f[20]), f[21]);
  const T smf4 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(f[1], f[2]), f[8]), f[9]), f[11]), f[16]), f[20]), f[21]);
  const T smf5 = rn_add(rn_add(rn_add(rn_add(rn_add(f[5], f[11]), f[14]), f[16]), f[20]), f[21]);
  const T smf6 = rn_add(rn_add(rn_add(rn_add(rn_add(f[4], f[8]), f[9]), f[14]), f[20]), f[21]);
  const T smf7 = rn_sub(rn_add(rn_add((-f[8]), f[9]), f[20]), f[21]);
  const T smf8 = rn_add(rn_sub(rn_sub(f[11], f[16]), f[20]), f[21]);
  const T smf9 = rn_sub(rn_sub(rn_sub((-f[11]), f[16]), f[20]), f[21]);
  const T smf10 = rn_add(rn_add(rn_add(f[8], f[9]), f[20]), f[21]);
  const T smf11 = rn_sub(rn_add(rn_add((-f[11]), f[16]), f[20]), f[21]);
  const T smf12 = rn_sub(rn_add(rn_add((-f[8]), f[9]), f[20]), f[21]);
  const T smf13 = rn_add(rn_add(rn_add(f[8], f[9]), f[20]), f[21]);
  const T smf14 = rn_add(rn_add(rn_add(f[11], f[16]), f[20]), f[21]);
  const T m0 = rho;
  const T m1 = rn_mul(rho, ux);
  const T m2 = rn_mul(rho, uy);
  const T m3 = rn_mul(rho, uz);
  const T m4 = rn_add(rn_mul((T(1) / T(3)), rho), rn_mul(rn_mul(rho, ux), ux));
  const T m5 = rn_add(rn_mul((T(1) / T(3)), rho), rn_mul(rn_mul(rho, uy), uy));
  const T m6 = rn_add(rn_mul((T(1) / T(3)), rho), rn_mul(rn_mul(rho, uz), uz));
  const T m7 = rn_mul(rn_mul(rho, ux), uz);
  const T m8 = rn_mul(rn_mul(rho, ux), uy);
  const T m9 = rn_add(rn_mul(rn_mul((T(1) / T(3)), rho), uy), rn_mul(rn_mul(rn_mul(rho, ux), ux), uy));
  const T m10 = rn_add(rn_mul(rn_mul((T(1) / T(3)), rho), uz), rn_mul(rn_mul(rn_mul(rho, ux), ux), uz));
  const T m11 = rn_add(rn_mul(rn_mul((T(1) / T(3)), rho), ux), rn_mul(rn_mul(rn_mul(rho, ux), uy), uy));
  const T m12 = rn_add(rn_mul(rn_mul((T(1) / T(3)), rho), ux), rn_mul(rn_mul(rn_mul(rho, ux), uz), uz));
  const T m13 = rn_add(rn_add(rn_add(rn_mul((T(1) / T(9)), rho), rn_mul(rn_mul(rn_mul((T(1) / T(3)), rho), ux), ux)), rn_mul(rn_mul(rn_mul((T(1) / T(3)), rho), uz), uz)), rn_mul(rn_mul(rn_mul(rn_mul(rho, ux), ux), uz), uz));
  const T m14 = rn_add(rn_add(rn_add(rn_mul((T(1) / T(9)), rho), rn_mul(rn_mul(rn_mul((T(1) / T(3)), rho), ux), ux)), rn_mul(rn_mul(rn_mul((T(1) / T(3)), rho), uy), uy)), rn_mul(rn_mul(rn_mul(rn_mul(rho, ux), ux), uy), uy));
  const T s0 = rn_sub(m0, smf0);
  const T s1 = rn_sub(m1, smf1);
  const T s2 = rn_sub(m2, smf2);
  const T s3 = rn_sub(m3, smf3);
  const T s4 = rn_sub(m4, smf4);
  const T s5 = rn_sub(m5, smf5);
  const T s6 = rn_sub(m6, smf6);
  const T s7 = rn_sub(m7, smf7);
  const T s8 = rn_sub(m8, smf8);
  const T s9 = rn_sub(m9, smf9);
  const T s10 = rn_sub(m10, smf10);
  const T s11 = rn_sub(m11, smf11);
  const T s12 = rn_sub(m12, smf12);
  const T s13 = rn_sub(m13, smf13);
  const T s14 = rn_sub(m14, smf14);
  f[3] = rn_add(rn_sub(rn_sub(s0, s4), s5), s14);
  f[6] = rn_add(rn_sub(rn_sub(s0, s4), s6), s13);
  f[7] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), s1), rn_mul((T(1) / T(2)), s4)), rn_mul((T(-1) / T(2)), s11)), rn_mul((T(-1) / T(2)), s14));
  f[10] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(2)), s1), rn_mul((T(1) / T(2)), s4)), rn_mul((T(1) / T(2)), s11)), rn_mul((T(-1) / T(2)), s14));
  f[12] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), s1), rn_mul((T(1) / T(2)), s4)), rn_mul((T(-1) / T(2)), s12)), rn_mul((T(-1) / T(2)), s13));
  f[13] = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add((-s0), rn_mul((T(1) / T(2)), s2)), rn_mul((T(-1) / T(2)), s3)), s4), rn_mul((T(1) / T(2)), s5)), rn_mul((T(1) / T(2)), s6)), rn_mul((T(-1) / T(2)), s9)), rn_mul((T(1) / T(2)), s10)), rn_mul((T(-1) / T(2)), s13)), rn_mul((T(-1) / T(2)), s14));
  f[15] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(2)), s1), rn_mul((T(1) / T(2)), s4)), rn_mul((T(1) / T(2)), s12)), rn_mul((T(-1) / T(2)), s13));
  f[17] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), s3), rn_mul((T(1) / T(2)), s6)), rn_mul((T(-1) / T(2)), s10)), rn_mul((T(-1) / T(2)), s13));
  f[18] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(2)), s2), rn_mul((T(1) / T(2)), s5)), rn_mul((T(1) / T(2)), s9)), rn_mul((T(-1) / T(2)), s14));
  f[19] = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), s1), rn_mul((T(-1) / T(2)), s4)), rn_mul((T(1) / T(4)), s7)), rn_mul((T(-1) / T(4)), s8)), rn_mul((T(1) / T(4)), s9)), rn_mul((T(-1) / T(4)), s10)), rn_mul((T(-1) / T(4)), s11)), rn_mul((T(-1) / T(4)), s12)), rn_mul((T(1) / T(4)), s13)), rn_mul((T(1) / T(4)), s14));
  f[22] = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_mul((T(-1) / T(2)), s1), rn_mul((T(-1) / T(2)), s4)), rn_mul((T(-1) / T(4)), s7)), rn_mul((T(1) / T(4)), s8)), rn_mul((T(1) / T(4)), s9)), rn_mul((T(-1) / T(4)), s10)), rn_mul((T(1) / T(4)), s11)), rn_mul((T(1) / T(4)), s12)), rn_mul((T(1) / T(4)), s13)), rn_mul((T(1) / T(4)), s14));
  f[23] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(4)), s8), rn_mul((T(-1) / T(4)), s9)), rn_mul((T(1) / T(4)), s11)), rn_mul((T(1) / T(4)), s14));
  f[24] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(4)), s7), rn_mul((T(1) / T(4)), s10)), rn_mul((T(-1) / T(4)), s12)), rn_mul((T(1) / T(4)), s13));
  f[25] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(4)), s8), rn_mul((T(-1) / T(4)), s9)), rn_mul((T(-1) / T(4)), s11)), rn_mul((T(1) / T(4)), s14));
  f[26] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(4)), s7), rn_mul((T(1) / T(4)), s10)), rn_mul((T(1) / T(4)), s12)), rn_mul((T(1) / T(4)), s13));
}
template <typename T>
PSL_HDI void restore_rho_u_n11(const T (&f)[27], T& rho, T& ux, T& uy, T& uz) {
  const T q0 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_mul(T(2), f[0]), rn_mul(T(2), f[1])), rn_mul(T(2), f[2])), f[4]), f[5]), f[8]), f[9]), f[11]), rn_mul(T(-4), f[14])), f[16]), rn_mul(T(-4), f[20])), rn_mul(T(-4), f[21]));
  const T q1 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_sub(f[1], f[2]), rn_mul(T(-2), f[8])), rn_mul(T(2), f[9])), rn_mul(T(-2), f[11])), rn_mul(T(2), f[16])), rn_mul(T(4), f[20])), rn_mul(T(-4), f[21]));
  const T q2 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), f[0]), rn_mul((T(1) / T(2)), f[1])), rn_mul((T(1) / T(2)), f[2])), f[4]), rn_mul(T(-2), f[5])), f[8]), f[9]), rn_mul(T(-2), f[11])), rn_mul(T(-4), f[14])), rn_mul(T(-2), f[16])), rn_mul(T(-4), f[20])), rn_mul(T(-4), f[21]));
  const T q3 = rn_add(rn_add(rn_sub(rn_add(rn_sub(rn_add(rn_add(rn_sub(rn_add(rn_add(rn_add(rn_mul((T(-1) / T(2)), f[0]), rn_mul((T(-1) / T(2)), f[1])), rn_mul((T(-1) / T(2)), f[2])), rn_mul(T(2), f[4])), f[5]), rn_mul(T(2), f[8])), rn_mul(T(2), f[9])), f[11]), rn_mul(T(4), f[14])), f[16]), rn_mul(T(4), f[20])), rn_mul(T(4), f[21]));
  rho = q0;
  ux = rn_div(q1, rho);
  uy = rn_div(q2, rho);
  uz = rn_div(q3, rho);
}
template <typename T>
PSL_HDI void restore_u_n11(const T (&f)[27], const T rho, T& ux, T& uy, T& uz) {
  const T scmf0 = rn_div(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_sub(rn_sub((-f[0]), f[1]), f[2]), rn_mul(T(-2), f[4])), rn_mul(T(-2), f[5])), rn_mul(T(-2), f[8])), rn_mul(T(-2), f[9])), rn_mul(T(-2), f[11])), rn_mul(T(-4), f[14])), rn_mul(T(-2), f[16])), rn_mul(T(-4), f[20])), rn_mul(T(-4), f[21])), rho);
  const T scmf1 = rn_div(rn_add(rn_add(rn_add(rn_sub(rn_sub((-f[0]), f[1]), f[2]), rn_mul(T(-2), f[4])), rn_mul(T(-2), f[8])), rn_mul(T(-2), f[9])), rho);
  const T scmf2 = rn_div(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add((-f[1]), f[2]), rn_mul(T(2), f[8])), rn_mul(T(-2), f[9])), rn_mul(T(2), f[11])), rn_mul(T(-2), f[16])), rn_mul(T(-4), f[20])), rn_mul(T(4), f[21])), rho);
  const T s0 = rn_sub(scmf0, T(-1));
  const T s1 = rn_sub(scmf1, (T(-2) / T(3)));
  const T s2 = rn_sub(scmf2, T(0));
  ux = (-s2);
  uy = rn_add(s0, rn_mul((T(-3) / T(2)), s1));
  uz = rn_mul((T(-3) / T(2)), s1);
}
template <typename T>
PSL_HDI void restore_rho_n11(const T (&f)[27], T& rho, const T ux, const T uy, const T uz) {
  const T scqu = rn_add(rn_mul(T(1), uy), rn_mul(T(-1), uz));
  const T s = rn_add(T(-1), scqu);
  const T scmf = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_sub(rn_sub((-f[0]), f[1]), f[2]), rn_mul(T(-2), f[4])), rn_mul(T(-2), f[5])), rn_mul(T(-2), f[8])), rn_mul(T(-2), f[9])), rn_mul(T(-2), f[11])), rn_mul(T(-4), f[14])), rn_mul(T(-2), f[16])), rn_mul(T(-4), f[20])), rn_mul(T(-4), f[21]));
  rho = rn_div(scmf, s);
}
template <typename T>
PSL_HDI void mirror_n11(T (&f)[27]) {
  f[3] = f[4];
  f[6] = f[5];
  f[7] = f[9];
  f[10] = f[8];
  f[12] = f[16];
  f[13] = f[14];
  f[15] = f[11];
  f[17] = f[14];
  f[18] = f[14];
  f[19] = f[21];
  f[22] = f[20];
  f[23] = f[20];
  f[24] = f[21];
  f[25] = f[21];
  f[26] = f[20];
}

// ---- outer normal (-1,+0,+1): 15 unknown populations ----
template <typename T>
PSL_HDI void mbbc_n5(T (&f)[27], const T rho, const T ux, const T uy, const T uz) {
  const T smf0 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(f[0], f[2]), f[4]), f[5]), f[6]), f[8]), f[11]), f[14]), f[15]), f[17]), f[21]), f[24]);
  const T smf1 = rn_sub(rn_sub(rn_sub(rn_sub(rn_sub((-f[2]), f[8]), f[11]), f[15]), f[21]), f[24]);
  const T smf2 = rn_add(rn_sub(rn_add(rn_add(rn_sub(rn_sub(rn_add((-f[5]), f[6]), f[11]), f[14]), f[15]), f[17]), f[21]), f[24]);
  const T smf3 = rn_add(rn_add(rn_add(rn_add(rn_add(f[4], f[8]), f[14]), f[17]), f[21]), f[24]);
  const T smf4 = rn_add(rn_add(rn_add(rn_add(rn_add(f[2], f[8]), f[11]), f[15]), f[21]), f[24]);
  const T smf5 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(f[5], f[6]), f[11]), f[14]), f[15]), f[17]), f[21]), f[24]);
  const T smf6 = rn_add(rn_add(rn_add(rn_add(rn_add(f[4], f[8]), f[14]), f[17]), f[21]), f[24]);
  const T smf7 = rn_add(rn_sub(rn_add((-f[14]), f[17]), f[21]), f[24]);
  const T smf8 = rn_sub(rn_add(rn_sub(f[11], f[15]), f[21]), f[24]);
  const T smf9 = rn_add(rn_sub(rn_add((-f[11]), f[15]), f[21]), f[24]);
  const T smf10 = rn_sub(rn_sub(rn_sub((-f[11]), f[15]), f[21]), f[24]);
  const T smf11 = rn_add(rn_add(rn_add(f[14], f[17]), f[21]), f[24]);
  const T smf12 = rn_add(rn_sub(rn_add((-f[14]), f[17]), f[21]), f[24]);
  const T smf13 = rn_add(rn_add(rn_add(f[14], f[17]), f[21]), f[24]);
  const T smf14 = rn_add(rn_add(rn_add(f[11], f[15]), f[21]), f[24]);
  const T m0 = rho;
  const T m1 = rn_mul(rho, ux);
  const T m2 = rn_mul(rho, uy);
  const T m3 = rn_mul(rho, uz);
  const T m4 = rn_add(rn_mul((T(1) / T(3)), rho), rn_mul(rn_mul(rho, ux), ux));
  const T m5 = rn_add(rn_mul((T(1) / T(3)), rho), rn_mul(rn_mul(rho, uy), uy));
  const T m6 = rn_add(rn_mul((T(1) / T(3)), rho), rn_mul(rn_mul(rho, uz), uz));
  const T m7 = rn_mul(rn_mul(rho, uy), uz);
  const T m8 = rn_mul(rn_mul(rho, ux), uy);
  const T m9 = rn_add(rn_mul(rn_mul((T(1) / T(3)), rho), uy), rn_mul(rn_mul(rn_mul(rho, ux), ux), uy));
  const T m10 = rn_add(rn_mul(rn_mul((T(1) / T(3)), rho), ux), rn_mul(rn_mul(rn_mul(rho, ux), uy), uy));
  const T m11 = rn_add(rn_mul(rn_mul((T(1) / T(3)), rho), uz), rn_mul(rn_mul(rn_mul(rho, uy), uy), uz));
  const T m12 = rn_add(rn_mul(rn_mul((T(1) / T(3)), rho), uy), rn_mul(rn_mul(rn_mul(rho, uy), uz), uz));
  const T m13 = rn_add(rn_add(rn_add(rn_mul((T(1) / T(9)), rho), rn_mul(rn_mul(rn_mul((T(1) / T(3)), rho), uy), uy)), rn_mul(rn_mul(rn_mul((T(1) / T(3)), rho), uz), uz)), rn_mul(rn_mul(rn_mul(rn_mul(rho, uy), uy), uz), uz));
  const T m14 = rn_add(rn_add(rn_add(rn_mul((T(1) / T(9)), rho), rn_mul(rn_mul(rn_mul((T(1) / T(3)), rho), ux), ux)), rn_mul(rn_mul(rn_mul((T(1) / T(3)), rho), uy), uy)), rn_mul(rn_mul(rn_mul(rn_mul(rho, ux), ux), uy), uy));
  const T s0 = rn_sub(m0, smf0);
  const T s1 = rn_sub(m1, smf1);
  const T s2 = rn_sub(m2, smf2);
  const T s3 = rn_sub(m3, smf3);
  const T s4 = rn_sub(m4, smf4);
  const T s5 = rn_sub(m5, smf5);
  const T s6 = rn_sub(m6, smf6);
  const T s7 = rn_sub(m7, smf7);
  const T s8 = rn_sub(m8, smf8);
  const T s9 = rn_sub(m9, smf9);
  const T s10 = rn_sub(m10, smf10);
  const T s11 = rn_sub(m11, smf11);
  const T s12 = rn_sub(m12, smf12);
  const T s13 = rn_sub(m13, smf13);
  const T s14 = rn_sub(m14, smf14);
  f[1] = rn_add(rn_sub(rn_sub(s0, s5), s6), s13);
  f[3] = rn_add(rn_sub(rn_sub(s0, s4), s5), s14);
  f[7] = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add((-s0), rn_mul((T(1) / T(2)), s1)), rn_mul((T(-1) / T(2)), s3)), rn_mul((T(1) / T(2)), s4)), s5), rn_mul((T(1) / T(2)), s6)), rn_mul((T(-1) / T(2)), s10)), rn_mul((T(1) / T(2)), s11)), rn_mul((T(-1) / T(2)), s13)), rn_mul((T(-1) / T(2)), s14));
  f[9] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), s3), rn_mul((T(1) / T(2)), s6)), rn_mul((T(-1) / T(2)), s11)), rn_mul((T(-1) / T(2)), s13));
  f[10] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(2)), s1), rn_mul((T(1) / T(2)), s4)), rn_mul((T(1) / T(2)), s10)), rn_mul((T(-1) / T(2)), s14));
  f[12] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), s2), rn_mul((T(1) / T(2)), s5)), rn_mul((T(-1) / T(2)), s12)), rn_mul((T(-1) / T(2)), s13));
  f[13] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), s2), rn_mul((T(1) / T(2)), s5)), rn_mul((T(-1) / T(2)), s9)), rn_mul((T(-1) / T(2)), s14));
  f[16] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(2)), s2), rn_mul((T(1) / T(2)), s5)), rn_mul((T(1) / T(2)), s12)), rn_mul((T(-1) / T(2)), s13));
  f[18] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(2)), s2), rn_mul((T(1) / T(2)), s5)), rn_mul((T(1) / T(2)), s9)), rn_mul((T(-1) / T(2)), s14));
  f[19] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(4)), s8), rn_mul((T(1) / T(4)), s9)), rn_mul((T(-1) / T(4)), s10)), rn_mul((T(1) / T(4)), s14));
  f[20] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(4)), s7), rn_mul((T(1) / T(4)), s11)), rn_mul((T(-1) / T(4)), s12)), rn_mul((T(1) / T(4)), s13));
  f[22] = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_mul((T(-1) / T(2)), s2), rn_mul((T(-1) / T(2)), s5)), rn_mul((T(-1) / T(4)), s7)), rn_mul((T(1) / T(4)), s8)), rn_mul((T(1) / T(4)), s9)), rn_mul((T(1) / T(4)), s10)), rn_mul((T(-1) / T(4)), s11)), rn_mul((T(1) / T(4)), s12)), rn_mul((T(1) / T(4)), s13)), rn_mul((T(1) / T(4)), s14));
  f[23] = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), s2), rn_mul((T(-1) / T(2)), s5)), rn_mul((T(1) / T(4)), s7)), rn_mul((T(-1) / T(4)), s8)), rn_mul((T(-1) / T(4)), s9)), rn_mul((T(1) / T(4)), s10)), rn_mul((T(-1) / T(4)), s11)), rn_mul((T(-1) / T(4)), s12)), rn_mul((T(1) / T(4)), s13)), rn_mul((T(1) / T(4)), s14));
  f[25] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(4)), s8), rn_mul((T(-1) / T(4)), s9)), rn_mul((T(-1) / T(4)), s10)), rn_mul((T(1) / T(4)), s14));
  f[26] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(4)), s7), rn_mul((T(1) / T(4)), s11)), rn_mul((T(1) / T(4)), s12)), rn_mul((T(1) / T(4)), s13));
}
template <typename T>
PSL_HDI void restore_rho_u_n5(const T (&f)[27], T& rho, T& ux, T& uy, T& uz) {
  const T q0 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_mul(T(2), f[0]), f[2]), f[4]), rn_mul(T(2), f[5])), rn_mul(T(2), f[6])), rn_mul(T(-4), f[8])), f[11]), f[14]), f[15]), f[17]), rn_mul(T(-4), f[21])), rn_mul(T(-4), f[24]));
  const T q1 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), f[0]), rn_mul(T(-2), f[2])), f[4]), rn_mul((T(1) / T(2)), f[5])), rn_mul((T(1) / T(2)), f[6])), rn_mul(T(-4), f[8])), rn_mul(T(-2), f[11])), f[14]), rn_mul(T(-2), f[15])), f[17]), rn_mul(T(-4), f[21])), rn_mul(T(-4), f[24]));
  const T q2 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add((-f[5]), f[6]), rn_mul(T(-2), f[11])), rn_mul(T(-2), f[14])), rn_mul(T(2), f[15])), rn_mul(T(2), f[17])), rn_mul(T(-4), f[21])), rn_mul(T(4), f[24]));
  const T q3 = rn_add(rn_add(rn_add(rn_sub(rn_add(rn_sub(rn_add(rn_add(rn_add(rn_add(rn_sub(rn_mul((T(-1) / T(2)), f[0]), f[2]), rn_mul(T(2), f[4])), rn_mul((T(-1) / T(2)), f[5])), rn_mul((T(-1) / T(2)), f[6])), rn_mul(T(4), f[8])), f[11]), rn_mul(T(2), f[14])), f[15]), rn_mul(T(2), f[17])), rn_mul(T(4), f[21])), rn_mul(T(4), f[24]));
  rho = q0;
  ux = rn_div(q1, rho);
  uy = rn_div(q2, rho);
  uz = rn_div(q3, rho);
}
template <typename T>
PSL_HDI void restore_u_n5(const T (&f)[27], const T rho, T& ux, T& uy, T& uz) {
  const T scmf0 = rn_div(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_sub(rn_sub(rn_add(rn_add((-f[0]), rn_mul(T(-2), f[2])), rn_mul(T(-2), f[4])), f[5]), f[6]), rn_mul(T(-4), f[8])), rn_mul(T(-2), f[11])), rn_mul(T(-2), f[14])), rn_mul(T(-2), f[15])), rn_mul(T(-2), f[17])), rn_mul(T(-4), f[21])), rn_mul(T(-4), f[24])), rho);
  const T scmf1 = rn_div(rn_add(rn_add(rn_sub(rn_sub(rn_add((-f[0]), rn_mul(T(-2), f[4])), f[5]), f[6]), rn_mul(T(-2), f[14])), rn_mul(T(-2), f[17])), rho);
  const T scmf2 = rn_div(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_sub(f[5], f[6]), rn_mul(T(2), f[11])), rn_mul(T(2), f[14])), rn_mul(T(-2), f[15])), rn_mul(T(-2), f[17])), rn_mul(T(4), f[21])), rn_mul(T(-4), f[24])), rho);
  const T s0 = rn_sub(scmf0, T(-1));
  const T s1 = rn_sub(scmf1, (T(-2) / T(3)));
  const T s2 = rn_sub(scmf2, T(0));
  ux = rn_add(s0, rn_mul((T(-3) / T(2)), s1));
  uy = (-s2);
  uz = rn_mul((T(-3) / T(2)), s1);
}
template <typename T>
PSL_HDI void restore_rho_n5(const T (&f)[27], T& rho, const T ux, const T uy, const T uz) {
  const T scqu = rn_add(rn_mul(T(1), ux), rn_mul(T(-1), uz));
  const T s = rn_add(T(-1), scqu);
  const T scmf = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_sub(rn_sub(rn_add(rn_add((-f[0]), rn_mul(T(-2), f[2])), rn_mul(T(-2), f[4])), f[5]), f[6]), rn_mul(T(-4), f[8])), rn_mul(T(-2), f[11])), rn_mul(T(-2), f[14])), rn_mul(T(-2), f[15])), rn_mul(T(-2), f[17])), rn_mul(T(-4), f[21])), rn_mul(T(-4), f[24]));
  rho = rn_div(scmf, s);
}
template <typename T>
PSL_HDI void mirror_n5(T (&f)[27]) {
  f[1] = f[2];
  f[3] = f[4];
  f[7] = f[8];
  f[9] = f[8];
  f[10] = f[8];
  f[12] = f[15];
  f[13] = f[17];
  f[16] = f[11];
  f[18] = f[14];
  f[19] = f[24];
  f[20] = f[21];
  f[22] = f[24];
  f[23] = f[21];
  f[25] = f[21];
  f[26] = f[24];
}

// ---- outer normal (-1,+1,+0): 15 unknown populations ----
template <typename T>
PSL_HDI void mbbc_n7(T (&f)[27], const T rho, const T ux, const T uy, const T uz) {
  const T smf0 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(f[0], f[2]), f[3]), f[4]), f[6]), f[8]), f[10]), f[13]), f[15]), f[17]), f[19]), f[24]);
  const T smf1 = rn_sub(rn_sub(rn_sub(rn_sub(rn_sub((-f[2]), f[8]), f[10]), f[15]), f[19]), f[24]);
  const T smf2 = rn_add(rn_add(rn_add(rn_add(rn_add(f[6], f[13]), f[15]), f[17]), f[19]), f[24]);
  const T smf3 = rn_add(rn_sub(rn_add(rn_sub(rn_sub(rn_add(rn_add((-f[3]), f[4]), f[8]), f[10]), f[13]), f[17]), f[19]), f[24]);
  const T smf4 = rn_add(rn_add(rn_add(rn_add(rn_add(f[2], f[8]), f[10]), f[15]), f[19]), f[24]);
  const T smf5 = rn_add(rn_add(rn_add(rn_add(rn_add(f[6], f[13]), f[15]), f[17]), f[19]), f[24]);
  const T smf6 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(f[3], f[4]), f[8]), f[10]), f[13]), f[17]), f[19]), f[24]);
  const T smf7 = rn_add(rn_sub(rn_add((-f[13]), f[17]), f[19]), f[24]);
  const T smf8 = rn_sub(rn_add(rn_add((-f[8]), f[10]), f[19]), f[24]);
  const T smf9 = rn_add(rn_sub(rn_sub(f[8], f[10]), f[19]), f[24]);
  const T smf10 = rn_add(rn_sub(rn_add((-f[13]), f[17]), f[19]), f[24]);
  const T smf11 = rn_sub(rn_sub(rn_sub((-f[8]), f[10]), f[19]), f[24]);
  const T smf12 = rn_add(rn_add(rn_add(f[13], f[17]), f[19]), f[24]);
  const T smf13 = rn_add(rn_add(rn_add(f[13], f[17]), f[19]), f[24]);
  const T smf14 = rn_add(rn_add(rn_add(f[8], f[10]), f[19]), f[24]);
  const T m0 = rho;
  const T m1 = rn_mul(rho, ux);
  const T m2 = rn_mul(rho, uy);
  const T m3 = rn_mul(rho, uz);
  const T m4 = rn_add(rn_mul((T(1) / T(3)), rho), rn_mul(rn_mul(rho, ux), ux));
  const T m5 = rn_add(rn_mul((T(1) / T(3)), rho), rn_mul(rn_mul(rho, uy), uy));
  const T m6 = rn_add(rn_mul((T(1) / T(3)), rho), rn_mul(rn_mul(rho, uz), uz));
  const T m7 = rn_mul(rn_mul(rho, uy), uz);
  const T m8 = rn_mul(rn_mul(rho, ux), uz);
  const T m9 = rn_add(rn_mul(rn_mul((T(1) / T(3)), rho), uz), rn_mul(rn_mul(rn_mul(rho, ux), ux), uz));
  const T m10 = rn_add(rn_mul(rn_mul((T(1) / T(3)), rho), uz), rn_mul(rn_mul(rn_mul(rho, uy), uy), uz));
  const T m11 = rn_add(rn_mul(rn_mul((T(1) / T(3)), rho), ux), rn_mul(rn_mul(rn_mul(rho, ux), uz), uz));
  const T m12 = rn_add(rn_mul(rn_mul((T(1) / T(3)), rho), uy), rn_mul(rn_mul(rn_mul(rho, uy), uz), uz));
  const T m13 = rn_add(rn_add(rn_add(rn_mul((T(1) / T(9)), rho), rn_mul(rn_mul(rn_mul((T(1) / T(3)), rho), uy), uy)), rn_mul(rn_mul(rn_mul((T(1) / T(3)), rho), uz), uz)), rn_mul(rn_mul(rn_mul(rn_mul(rho, uy), uy), uz), uz));
  const T m14 = rn_add(rn_add(rn_add(rn_mul((T(1) / T(9)), rho), rn_mul(rn_mul(rn_mul((T(1) / T(3)), rho), ux), ux)), rn_mul(rn_mul(rn_mul((T(1) / T(3)), rho), uz), uz)), rn_mul(rn_mul(rn_mul(rn_mul(rho, ux), ux), uz), uz));
  const T s0 = rn_sub(m0, smf0);
  const T s1 = rn_sub(m1, smf1);
  const T s2 = rn_sub(m2, smf2);
  const T s3 = rn_sub(m3, smf3);
  const T s4 = rn_sub(m4, smf4);
  const T s5 = rn_sub(m5, smf5);
  const T s6 = rn_sub(m6, smf6);
  const T s7 = rn_sub(m7, smf7);
  const T s8 = rn_sub(m8, smf8);
  const T s9 = rn_sub(m9, smf9);
  const T s10 = rn_sub(m10, smf10);
  const T s11 = rn_sub(m11, smf11);
  const T s12 = rn_sub(m12, smf12);
  const T s13 = rn_sub(m13, smf13);
  const T s14 = rn_sub(m14, smf14);
  f[1] = rn_add(rn_sub(rn_sub(s0, s5), s6), s13);
  f[5] = rn_add(rn_sub(rn_sub(s0, s4), s6), s14);
  f[7] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(2)), s3), rn_mul((T(1) / T(2)), s6)), rn_mul((T(1) / T(2)), s10)), rn_mul((T(-1) / T(2)), s13));
  f[9] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), s3), rn_mul((T(1) / T(2)), s6)), rn_mul((T(-1) / T(2)), s10)), rn_mul((T(-1) / T(2)), s13));
  f[11] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(2)), s1), rn_mul((T(1) / T(2)), s4)), rn_mul((T(1) / T(2)), s11)), rn_mul((T(-1) / T(2)), s14));
  f[12] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), s2), rn_mul((T(1) / T(2)), s5)), rn_mul((T(-1) / T(2)), s12)), rn_mul((T(-1) / T(2)), s13));
  f[14] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), s3), rn_mul((T(1) / T(2)), s6)), rn_mul((T(-1) / T(2)), s9)), rn_mul((T(-1) / T(2)), s14));
  f[16] = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add((-s0), rn_mul((T(1) / T(2)), s1)), rn_mul((T(-1) / T(2)), s2)), rn_mul((T(1) / T(2)), s4)), rn_mul((T(1) / T(2)), s5)), s6), rn_mul((T(-1) / T(2)), s11)), rn_mul((T(1) / T(2)), s12)), rn_mul((T(-1) / T(2)), s13)), rn_mul((T(-1) / T(2)), s14));
  f[18] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(2)), s3), rn_mul((T(1) / T(2)), s6)), rn_mul((T(1) / T(2)), s9)), rn_mul((T(-1) / T(2)), s14));
  f[20] = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_mul((T(-1) / T(2)), s3), rn_mul((T(-1) / T(2)), s6)), rn_mul((T(-1) / T(4)), s7)), rn_mul((T(1) / T(4)), s8)), rn_mul((T(1) / T(4)), s9)), rn_mul((T(1) / T(4)), s10)), rn_mul((T(1) / T(4)), s11)), rn_mul((T(-1) / T(4)), s12)), rn_mul((T(1) / T(4)), s13)), rn_mul((T(1) / T(4)), s14));
  f[21] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(4)), s8), rn_mul((T(1) / T(4)), s9)), rn_mul((T(-1) / T(4)), s11)), rn_mul((T(1) / T(4)), s14));
  f[22] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(4)), s7), rn_mul((T(-1) / T(4)), s10)), rn_mul((T(1) / T(4)), s12)), rn_mul((T(1) / T(4)), s13));
  f[23] = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), s3), rn_mul((T(-1) / T(2)), s6)), rn_mul((T(1) / T(4)), s7)), rn_mul((T(-1) / T(4)), s8)), rn_mul((T(-1) / T(4)), s9)), rn_mul((T(-1) / T(4)), s10)), rn_mul((T(1) / T(4)), s11)), rn_mul((T(-1) / T(4)), s12)), rn_mul((T(1) / T(4)), s13)), rn_mul((T(1) / T(4)), s14));
  f[25] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(4)), s8), rn_mul((T(-1) / T(4)), s9)), rn_mul((T(-1) / T(4)), s11)), rn_mul((T(1) / T(4)), s14));
  f[26] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(4)), s7), rn_mul((T(1) / T(4)), s10)), rn_mul((T(1) / T(4)), s12)), rn_mul((T(1) / T(4)), s13));
}
template <typename T>
PSL_HDI void restore_rho_u_n7(const T (&f)[27], T& rho, T& ux, T& uy, T& uz) {
  const T q0 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_mul(T(2), f[0]), f[2]), rn_mul(T(2), f[3])), rn_mul(T(2), f[4])), f[6]), f[8]), f[10]), f[13]), rn_mul(T(-4), f[15])), f[17]), rn_mul(T(-4), f[19])), rn_mul(T(-4), f[24]));
  const T q1 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), f[0]), rn_mul(T(-2), f[2])), rn_mul((T(1) / T(2)), f[3])), rn_mul((T(1) / T(2)), f[4])), f[6]), rn_mul(T(-2), f[8])), rn_mul(T(-2), f[10])), f[13]), rn_mul(T(-4), f[15])), f[17]), rn_mul(T(-4), f[19])), rn_mul(T(-4), f[24]));
  const T q2 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_sub(rn_sub(rn_add(rn_add(rn_add(rn_sub(rn_mul((T(-1) / T(2)), f[0]), f[2]), rn_mul((T(-1) / T(2)), f[3])), rn_mul((T(-1) / T(2)), f[4])), rn_mul(T(2), f[6])), f[8]), f[10]), rn_mul(T(2), f[13])), rn_mul(T(4), f[15])), rn_mul(T(2), f[17])), rn_mul(T(4), f[19])), rn_mul(T(4), f[24]));
  const T q3 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add((-f[3]), f[4]), rn_mul(T(2), f[8])), rn_mul(T(-2), f[10])), rn_mul(T(-2), f[13])), rn_mul(T(2), f[17])), rn_mul(T(-4), f[19])), rn_mul(T(4), f[24]));
  rho = q0;
  ux = rn_div(q1, rho);
  uy = rn_div(q2, rho);
  uz = rn_div(q3, rho);
}
template <typename T>
PSL_HDI void restore_u_n7(const T (&f)[27], const T rho, T& ux, T& uy, T& uz) {
  const T scmf0 = rn_div(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_sub(rn_sub(rn_add((-f[0]), rn_mul(T(-2), f[2])), f[3]), f[4]), rn_mul(T(-2), f[6])), rn_mul(T(-2), f[8])), rn_mul(T(-2), f[10])), rn_mul(T(-2), f[13])), rn_mul(T(-4), f[15])), rn_mul(T(-2), f[17])), rn_mul(T(-4), f[19])), rn_mul(T(-4), f[24])), rho);
  const T scmf1 = rn_div(rn_add(rn_add(rn_add(rn_sub(rn_sub((-f[0]), f[3]), f[4]), rn_mul(T(-2), f[6])), rn_mul(T(-2), f[13])), rn_mul(T(-2), f[17])), rho);
  const T scmf2 = rn_div(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_sub(f[3], f[4]), rn_mul(T(-2), f[8])), rn_mul(T(2), f[10])), rn_mul(T(2), f[13])), rn_mul(T(-2), f[17])), rn_mul(T(4), f[19])), rn_mul(T(-4), f[24])), rho);
  const T s0 = rn_sub(scmf0, T(-1));
  const T s1 = rn_sub(scmf1, (T(-2) / T(3)));
  const T s2 = rn_sub(scmf2, T(0));
  ux = rn_add(s0, rn_mul((T(-3) / T(2)), s1));
  uy = rn_mul((T(-3) / T(2)), s1);
  uz = (-s2);
}
template <typename T>
PSL_HDI void restore_rho_n7(const T (&f)[27], T& rho, const T ux, const T uy, const T uz) {
  const T scqu = rn_add(rn_mul(T(1), ux), rn_mul(T(-1), uy));
  const T s = rn_add(T(-1), scqu);
  const T scmf = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_sub(rn_sub(rn_add((-f[0]), rn_mul(T(-2), f[2])), f[3]), f[4]), rn_mul(T(-2), f[6])), rn_mul(T(-2), f[8])), rn_mul(T(-2), f[10])), rn_mul(T(-2), f[13])), rn_mul(T(-4), f[15])), rn_mul(T(-2), f[17])), rn_mul(T(-4), f[19])), rn_mul(T(-4), f[24]));
  rho = rn_div(scmf, s);
}
template <typename T>
PSL_HDI void mirror_n7(T (&f)[27]) {
  f[1] = f[2];
  f[5] = f[6];
  f[7] = f[10];
  f[9] = f[8];
  f[11] = f[15];
  f[12] = f[15];
  f[14] = f[17];
  f[16] = f[15];
  f[18] = f[13];
  f[20] = f[24];
  f[21] = f[24];
  f[22] = f[19];
  f[23] = f[19];
  f[25] = f[19];
  f[26] = f[24];
}

// ---- outer normal (+1,+1,+1): 19 unknown populations ----
template <typename T>
PSL_HDI void mbbc_n26(T (&f)[27], const T rho, const T ux, const T uy, const T uz) {
  const T smf0 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(f[0], f[1]), f[4]), f[6]), f[9]), f[12]), f[17]), f[26]);
  const T smf1 = rn_add(rn_add(rn_add(f[1], f[9]), f[12]), f[26]);
  const T smf2 = rn_add(rn_add(rn_add(f[6], f[12]), f[17]), f[26]);
  const T smf3 = rn_add(rn_add(rn_add(f[4], f[9]), f[17]), f[26]);
  const T smf4 = rn_add(rn_add(rn_add(f[1], f[9]), f[12]), f[26]);
  const T smf5 = rn_add(rn_add(rn_add(f[6], f[12]), f[17]), f[26]);
  const T smf6 = rn_add(rn_add(rn_add(f[4], f[9]), f[17]), f[26]);
  const T smf7 = rn_add(f[17], f[26]);
  const T smf8 = rn_add(f[9], f[26]);
  const T smf9 = rn_add(f[12], f[26]);
  const T smf10 = rn_add(f[12], f[26]);
  const T smf11 = rn_add(f[9], f[26]);
  const T smf12 = rn_add(f[12], f[26]);
  const T smf13 = rn_add(f[17], f[26]);
  const T smf14 = rn_add(f[9], f[26]);
  const T smf15 = rn_add(f[17], f[26]);
  const T smf16 = rn_add(f[17], f[26]);
  const T smf17 = rn_add(f[9], f[26]);
  const T smf18 = rn_add(f[12], f[26]);
  const T m0 = rho;
  const T m1 = rn_mul(rho, ux);
  const T m2 = rn_mul(rho, uy);
  const T m3 = rn_mul(rho, uz);
  const T m4 = rn_add(rn_mul((T(1) / T(3)), rho), rn_mul(rn_mul(rho, ux), ux));
  const T m5 = rn_add(rn_mul((T(1) / T(3)), rho), rn_mul(rn_mul(rho, uy), uy));
  const T m6 = rn_add(rn_mul((T(1) / T(3)), rho), rn_mul(rn_mul(rho, uz), uz));
  const T m7 = rn_mul(rn_mul(rho, uy), uz);
  const T m8 = rn_mul(rn_mul(rho, ux), uz);
  const T m9 = rn_mul(rn_mul(rho, ux), uy);
  const T m10 = rn_add(rn_mul(rn_mul((T(1) / T(3)), rho), uy), rn_mul(rn_mul(rn_mul(rho, ux), ux), uy));
  const T m11 = rn_add(rn_mul(rn_mul((T(1) / T(3)), rho), uz), rn_mul(rn_mul(rn_mul(rho, ux), ux), uz));
  const T m12 = rn_add(rn_mul(rn_mul((T(1) / T(3)), rho), ux), rn_mul(rn_mul(rn_mul(rho, ux), uy), uy));
  const T m13 = rn_add(rn_mul(rn_mul((T(1) / T(3)), rho), uz), rn_mul(rn_mul(rn_mul(rho, uy), uy), uz));
  const T m14 = rn_add(rn_mul(rn_mul((T(1) / T(3)), rho), ux), rn_mul(rn_mul(rn_mul(rho, ux), uz), uz));
  const T m15 = rn_add(rn_mul(rn_mul((T(1) / T(3)), rho), uy), rn_mul(rn_mul(rn_mul(rho, uy), uz), uz));
  const T m16 = rn_add(rn_add(rn_add(rn_mul((T(1) / T(9)), rho), rn_mul(rn_mul(rn_mul((T(1) / T(3)), rho), uy), uy)), rn_mul(rn_mul(rn_mul((T(1) / T(3)), rho), uz), uz)), rn_mul(rn_mul(rn_mul(rn_mul(rho, uy), uy), uz), uz));
  const T m17 = rn_add(rn_add(rn_add(rn_mul((T(1) / T(9)), rho), rn_mul(rn_mul(rn_mul((T(1) / T(3)), rho), ux), ux)), rn_mul(rn_mul(rn_mul((T(1) / T(3)), rho), uz), uz)), rn_mul(rn_mul(rn_mul(rn_mul(rho, ux), ux), uz), uz));
  const T m18 = rn_add(rn_add(rn_add(rn_mul((T(1) / T(9)), rho), rn_mul(rn_mul(rn_mul((T(1) / T(3)), rho), ux), ux)), rn_mul(rn_mul(rn_mul((T(1) / T(3)), rho), uy), uy)), rn_mul(rn_mul(rn_mul(rn_mul(rho, ux), ux), uy), uy));
  const T s0 = rn_sub(m0, smf0);
  const T s1 = rn_sub(m1, smf1);
  const T s2 = rn_sub(m2, smf2);
  const T s3 = rn_sub(m3, smf3);
  const T s4 = rn_sub(m4, smf4);
  const T s5 = rn_sub(m5, smf5);
  const T s6 = rn_sub(m6, smf6);
  const T s7 = rn_sub(m7, smf7);
  const T s8 = rn_sub(m8, smf8);
  const T s9 = rn_sub(m9, smf9);
  const T s10 = rn_sub(m10, smf10);
  const T s11 = rn_sub(m11, smf11);
  const T s12 = rn_sub(m12, smf12);
  const T s13 = rn_sub(m13, smf13);
  const T s14 = rn_sub(m14, smf14);
  const T s15 = rn_sub(m15, smf15);
  const T s16 = rn_sub(m16, smf16);
  const T s17 = rn_sub(m17, smf17);
  const T s18 = rn_sub(m18, smf18);
  f[2] = rn_add(rn_sub(rn_sub(s0, s5), s6), s16);
  f[3] = rn_add(rn_sub(rn_sub(s0, s4), s5), s18);
  f[5] = rn_add(rn_sub(rn_sub(s0, s4), s6), s17);
  f[7] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), s1), rn_mul((T(1) / T(2)), s4)), rn_mul((T(-1) / T(2)), s12)), rn_mul((T(-1) / T(2)), s18));
  f[8] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), s3), rn_mul((T(1) / T(2)), s6)), rn_mul((T(-1) / T(2)), s13)), rn_mul((T(-1) / T(2)), s16));
  f[10] = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add((-s0), rn_mul((T(-1) / T(2)), s1)), rn_mul((T(-1) / T(2)), s3)), rn_mul((T(1) / T(2)), s4)), s5), rn_mul((T(1) / T(2)), s6)), rn_mul((T(1) / T(2)), s12)), rn_mul((T(1) / T(2)), s13)), rn_mul((T(-1) / T(2)), s16)), rn_mul((T(-1) / T(2)), s18));
  f[11] = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add((-s0), rn_mul((T(-1) / T(2)), s1)), rn_mul((T(-1) / T(2)), s2)), rn_mul((T(1) / T(2)), s4)), rn_mul((T(1) / T(2)), s5)), s6), rn_mul((T(1) / T(2)), s14)), rn_mul((T(1) / T(2)), s15)), rn_mul((T(-1) / T(2)), s16)), rn_mul((T(-1) / T(2)), s17));
  f[13] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), s2), rn_mul((T(1) / T(2)), s5)), rn_mul((T(-1) / T(2)), s10)), rn_mul((T(-1) / T(2)), s18));
  f[14] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), s3), rn_mul((T(1) / T(2)), s6)), rn_mul((T(-1) / T(2)), s11)), rn_mul((T(-1) / T(2)), s17));
  f[15] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), s2), rn_mul((T(1) / T(2)), s5)), rn_mul((T(-1) / T(2)), s15)), rn_mul((T(-1) / T(2)), s16));
  f[16] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), s1), rn_mul((T(1) / T(2)), s4)), rn_mul((T(-1) / T(2)), s14)), rn_mul((T(-1) / T(2)), s17));
  f[18] = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add((-s0), rn_mul((T(-1) / T(2)), s2)), rn_mul((T(-1) / T(2)), s3)), s4), rn_mul((T(1) / T(2)), s5)), rn_mul((T(1) / T(2)), s6)), rn_mul((T(1) / T(2)), s10)), rn_mul((T(1) / T(2)), s11)), rn_mul((T(-1) / T(2)), s17)), rn_mul((T(-1) / T(2)), s18));
  f[19] = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_mul((T(-1) / T(2)), s2), rn_mul((T(-1) / T(2)), s5)), rn_mul((T(-1) / T(4)), s7)), rn_mul((T(-1) / T(4)), s9)), rn_mul((T(1) / T(4)), s10)), rn_mul((T(-1) / T(4)), s12)), rn_mul((T(-1) / T(4)), s13)), rn_mul((T(1) / T(4)), s15)), rn_mul((T(1) / T(4)), s16)), rn_mul((T(1) / T(4)), s18));
  f[20] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(4)), s8), rn_mul((T(1) / T(4)), s11)), rn_mul((T(1) / T(4)), s14)), rn_mul((T(1) / T(4)), s17));
  f[21] = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_mul((T(-1) / T(2)), s3), rn_mul((T(-1) / T(2)), s6)), rn_mul((T(-1) / T(4)), s7)), rn_mul((T(-1) / T(4)), s8)), rn_mul((T(1) / T(4)), s11)), rn_mul((T(1) / T(4)), s13)), rn_mul((T(-1) / T(4)), s14)), rn_mul((T(-1) / T(4)), s15)), rn_mul((T(1) / T(4)), s16)), rn_mul((T(1) / T(4)), s17));
  f[22] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(4)), s9), rn_mul((T(1) / T(4)), s10)), rn_mul((T(1) / T(4)), s12)), rn_mul((T(1) / T(4)), s18));
  f[23] = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_mul((T(-1) / T(2)), s1), rn_mul((T(-1) / T(2)), s4)), rn_mul((T(-1) / T(4)), s8)), rn_mul((T(-1) / T(4)), s9)), rn_mul((T(-1) / T(4)), s10)), rn_mul((T(-1) / T(4)), s11)), rn_mul((T(1) / T(4)), s12)), rn_mul((T(1) / T(4)), s14)), rn_mul((T(1) / T(4)), s17)), rn_mul((T(1) / T(4)), s18));
  f[24] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(4)), s7), rn_mul((T(1) / T(4)), s13)), rn_mul((T(1) / T(4)), s15)), rn_mul((T(1) / T(4)), s16));
  f[25] = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(s0, rn_mul((T(1) / T(2)), s1)), rn_mul((T(1) / T(2)), s2)), rn_mul((T(1) / T(2)), s3)), rn_mul((T(-1) / T(2)), s4)), rn_mul((T(-1) / T(2)), s5)), rn_mul((T(-1) / T(2)), s6)), rn_mul((T(1) / T(4)), s7)), rn_mul((T(1) / T(4)), s8)), rn_mul((T(1) / T(4)), s9)), rn_mul((T(-1) / T(4)), s10)), rn_mul((T(-1) / T(4)), s11)), rn_mul((T(-1) / T(4)), s12)), rn_mul((T(-1) / T(4)), s13)), rn_mul((T(-1) / T(4)), s14)), rn_mul((T(-1) / T(4)), s15)), rn_mul((T(1) / T(4)), s16)), rn_mul((T(1) / T(4)), s17)), rn_mul((T(1) / T(4)), s18));
}
template <typename T>
PSL_HDI void restore_rho_u_n26(const T (&f)[27], T& rho, T& ux, T& uy, T& uz) {
  const T q0 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_mul((T(5) / T(2)), f[0]), rn_mul(T(2), f[1])), rn_mul(T(2), f[4])), rn_mul(T(2), f[6])), rn_mul(T(-2), f[9])), rn_mul(T(-2), f[12])), rn_mul(T(-2), f[17])), rn_mul(T(-16), f[26]));
  const T q1 = rn_add(rn_add(rn_add(rn_add(rn_sub(rn_sub(rn_add(rn_mul((T(-1) / T(2)), f[0]), rn_mul(T(2), f[1])), f[4]), f[6]), rn_mul(T(4), f[9])), rn_mul(T(4), f[12])), rn_mul(T(-2), f[17])), rn_mul(T(8), f[26]));
  const T q2 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_sub(rn_sub(rn_mul((T(-1) / T(2)), f[0]), f[1]), f[4]), rn_mul(T(2), f[6])), rn_mul(T(-2), f[9])), rn_mul(T(4), f[12])), rn_mul(T(4), f[17])), rn_mul(T(8), f[26]));
  const T q3 = rn_add(rn_add(rn_add(rn_add(rn_sub(rn_add(rn_sub(rn_mul((T(-1) / T(2)), f[0]), f[1]), rn_mul(T(2), f[4])), f[6]), rn_mul(T(4), f[9])), rn_mul(T(-2), f[12])), rn_mul(T(4), f[17])), rn_mul(T(8), f[26]));
  rho = q0;
  ux = rn_div(q1, rho);
  uy = rn_div(q2, rho);
  uz = rn_div(q3, rho);
}
template <typename T>
PSL_HDI void restore_u_n26(const T (&f)[27], const T rho, T& ux, T& uy, T& uz) {
  const T scmf0 = rn_div(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(f[0], rn_mul(T(2), f[1])), rn_mul(T(2), f[4])), rn_mul(T(2), f[6])), rn_mul(T(4), f[9])), rn_mul(T(4), f[12])), rn_mul(T(4), f[17])), rn_mul(T(8), f[26])), rho);
  const T scmf1 = rn_div(rn_add(rn_add(rn_add((-f[0]), rn_mul(T(-2), f[4])), rn_mul(T(-2), f[6])), rn_mul(T(-4), f[17])), rho);
  const T scmf2 = rn_div(rn_add(rn_add(rn_add((-f[0]), rn_mul(T(-2), f[1])), rn_mul(T(-2), f[4])), rn_mul(T(-4), f[9])), rho);
  const T s0 = rn_sub(scmf0, T(1));
  const T s1 = rn_sub(scmf1, (T(-2) / T(3)));
  const T s2 = rn_sub(scmf2, (T(-2) / T(3)));
  ux = rn_add(s0, rn_mul((T(3) / T(2)), s1));
  uy = rn_add(s0, rn_mul((T(3) / T(2)), s2));
  uz = rn_add(rn_add((-s0), rn_mul((T(-3) / T(2)), s1)), rn_mul((T(-3) / T(2)), s2));
}
template <typename T>
PSL_HDI void restore_rho_n26(const T (&f)[27], T& rho, const T ux, const T uy, const T uz) {
  const T scqu = rn_add(rn_add(rn_mul(T(1), ux), rn_mul(T(1), uy)), rn_mul(T(1), uz));
  const T s = rn_add(T(1), scqu);
  const T scmf = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(f[0], rn_mul(T(2), f[1])), rn_mul(T(2), f[4])), rn_mul(T(2), f[6])), rn_mul(T(4), f[9])), rn_mul(T(4), f[12])), rn_mul(T(4), f[17])), rn_mul(T(8), f[26]));
  rho = rn_div(scmf, s);
}
template <typename T>
PSL_HDI void mirror_n26(T (&f)[27]) {
  f[2] = f[1];
  f[3] = f[4];
  f[5] = f[6];
  f[7] = f[9];
  f[8] = f[9];
  f[10] = f[9];
  f[11] = f[12];
  f[13] = f[17];
  f[14] = f[17];
  f[15] = f[12];
  f[16] = f[12];
  f[18] = f[17];
  f[19] = f[26];
  f[20] = f[26];
  f[21] = f[26];
  f[22] = f[26];
  f[23] = f[26];
  f[24] = f[26];
  f[25] = f[26];
}

// ---- outer normal (-1,-1,-1): 19 unknown populations ----
template <typename T>
PSL_HDI void mbbc_n0(T (&f)[27], const T rho, const T ux, const T uy, const T uz) {
  const T smf0 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(f[0], f[2]), f[3]), f[5]), f[10]), f[11]), f[18]), f[25]);
  const T smf1 = rn_sub(rn_sub(rn_sub((-f[2]), f[10]), f[11]), f[25]);
  const T smf2 = rn_sub(rn_sub(rn_sub((-f[5]), f[11]), f[18]), f[25]);
  const T smf3 = rn_sub(rn_sub(rn_sub((-f[3]), f[10]), f[18]), f[25]);
  const T smf4 = rn_add(rn_add(rn_add(f[2], f[10]), f[11]), f[25]);
  const T smf5 = rn_add(rn_add(rn_add(f[5], f[11]), f[18]), f[25]);
  const T smf6 = rn_add(rn_add(rn_add(f[3], f[10]), f[18]), f[25]);
  const T smf7 = rn_add(f[18], f[25]);
  const T smf8 = rn_add(f[10], f[25]);
  const T smf9 = rn_add(f[11], f[25]);
  const T smf10 = rn_sub((-f[11]), f[25]);
  const T smf11 = rn_sub((-f[10]), f[25]);
  const T smf12 = rn_sub((-f[11]), f[25]);
  const T smf13 = rn_sub((-f[18]), f[25]);
  const T smf14 = rn_sub((-f[10]), f[25]);
  const T smf15 = rn_sub((-f[18]), f[25]);
  const T smf16 = rn_add(f[18], f[25]);
  const T smf17 = rn_add(f[10], f[25]);
  const T smf18 = rn_add(f[11], f[25]);
  const T m0 = rho;
  const T m1 = rn_mul(rho, ux);
  const T m2 = rn_mul(rho, uy);
  const T m3 = rn_mul(rho, uz);
  const T m4 = rn_add(rn_mul((T(1) / T(3)), rho), rn_mul(rn_mul(rho, ux), ux));
  const T m5 = rn_add(rn_mul((T(1) / T(3)), rho), rn_mul(rn_mul(rho, uy), uy));
  const T m6 = rn_add(rn_mul((T(1) / T(3)), rho), rn_mul(rn_mul(rho, uz), uz));
  const T m7 = rn_mul(rn_mul(rho, uy), uz);
  const T m8 = rn_mul(rn_mul(rho, ux), uz);
  const T m9 = rn_mul(rn_mul(rho, ux), uy);
  const T m10 = rn_add(rn_mul(rn_mul((T(1) / T(3)), rho), uy), rn_mul(rn_mul(rn_mul(rho, ux), ux), uy));
  const T m11 = rn_add(rn_mul(rn_mul((T(1) / T(3)), rho), uz), rn_mul(rn_mul(rn_mul(rho, ux), ux), uz));
  const T m12 = rn_add(rn_mul(rn_mul((T(1) / T(3)), rho), ux), rn_mul(rn_mul(rn_mul(rho, ux), uy), uy));
  const T m13 = rn_add(rn_mul(rn_mul((T(1) / T(3)), rho), uz), rn_mul(rn_mul(rn_mul(rho, uy), uy), uz));
  const T m14 = rn_add(rn_mul(rn_mul((T(1) / T(3)), rho), ux), rn_mul(rn_mul(rn_mul(rho, ux), uz), uz));
  const T m15 = rn_add(rn_mul(rn_mul((T(1) / T(3)), rho), uy), rn_mul(rn_mul(rn_mul(rho, uy), uz), uz));
  const T m16 = rn_add(rn_add(rn_add(rn_mul((T(1) / T(9)), rho), rn_mul(rn_mul(rn_mul((T(1) / T(3)), rho), uy), uy)), rn_mul(rn_mul(rn_mul((T(1) / T(3)), rho), uz), uz)), rn_mul(rn_mul(rn_mul(rn_mul(rho, uy), uy), uz), uz));
  const T m17 = rn_add(rn_add(rn_add(rn_mul((T(1) / T(9)), rho), rn_mul(rn_mul(rn_mul((T(1) / T(3)), rho), ux), ux)), rn_mul(rn_mul(rn_mul((T(1) / T(3)), rho), uz), uz)), rn_mul(rn_mul(rn_mul(rn_mul(rho, ux), ux), uz), uz));
  const T m18 = rn_add(rn_add(rn_add(rn_mul((T(1) / T(9)), rho), rn_mul(rn_mul(rn_mul((T(1) / T(3)), rho), ux), ux)), rn_mul(rn_mul(rn_mul((T(1) / T(3)), rho), uy), uy)), rn_mul(rn_mul(rn_mul(rn_mul(rho, ux), ux), uy), uy));
  const T s0 = rn_sub(m0, smf0);
  const T s1 = rn_sub(m1, smf1);
  const T s2 = rn_sub(m2, smf2);
  const T s3 = rn_sub(m3, smf3);
  const T s4 = rn_sub(m4, smf4);
  const T s5 = rn_sub(m5, smf5);
  const T s6 = rn_sub(m6, smf6);
  const T s7 = rn_sub(m7, smf7);
  const T s8 = rn_sub(m8, smf8);
  const T s9 = rn_sub(m9, smf9);
  const T s10 = rn_sub(m10, smf10);
  const T s11 = rn_sub(m11, smf11);
  const T s12 = rn_sub(m12, smf12);
  const T s13 = rn_sub(m13, smf13);
  const T s14 = rn_sub(m14, smf14);
  const T s15 = rn_sub(m15, smf15);
  const T s16 = rn_sub(m16, smf16);
  const T s17 = rn_sub(m17, smf17);
  const T s18 = rn_sub(m18, smf18);
  f[1] = rn_add(rn_sub(rn_sub(s0, s5), s6), s16);
  f[4] = rn_add(rn_sub(rn_sub(s0, s4), s5), s18);
  f[6] = rn_add(rn_sub(rn_sub(s0, s4), s6), s17);
  f[7] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(2)), s3), rn_mul((T(1) / T(2)), s6)), rn_mul((T(1) / T(2)), s13)), rn_mul((T(-1) / T(2)), s16));
  f[8] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(2)), s1), rn_mul((T(1) / T(2)), s4)), rn_mul((T(1) / T(2)), s12)), rn_mul((T(-1) / T(2)), s18));
  f[9] = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add((-s0), rn_mul((T(1) / T(2)), s1)), rn_mul((T(1) / T(2)), s3)), rn_mul((T(1) / T(2)), s4)), s5), rn_mul((T(1) / T(2)), s6)), rn_mul((T(-1) / T(2)), s12)), rn_mul((T(-1) / T(2)), s13)), rn_mul((T(-1) / T(2)), s16)), rn_mul((T(-1) / T(2)), s18));
  f[12] = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add((-s0), rn_mul((T(1) / T(2)), s1)), rn_mul((T(1) / T(2)), s2)), rn_mul((T(1) / T(2)), s4)), rn_mul((T(1) / T(2)), s5)), s6), rn_mul((T(-1) / T(2)), s14)), rn_mul((T(-1) / T(2)), s15)), rn_mul((T(-1) / T(2)), s16)), rn_mul((T(-1) / T(2)), s17));
  f[13] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(2)), s3), rn_mul((T(1) / T(2)), s6)), rn_mul((T(1) / T(2)), s11)), rn_mul((T(-1) / T(2)), s17));
  f[14] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(2)), s2), rn_mul((T(1) / T(2)), s5)), rn_mul((T(1) / T(2)), s10)), rn_mul((T(-1) / T(2)), s18));
  f[15] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(2)), s1), rn_mul((T(1) / T(2)), s4)), rn_mul((T(1) / T(2)), s14)), rn_mul((T(-1) / T(2)), s17));
  f[16] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(2)), s2), rn_mul((T(1) / T(2)), s5)), rn_mul((T(1) / T(2)), s15)), rn_mul((T(-1) / T(2)), s16));
  f[17] = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add((-s0), rn_mul((T(1) / T(2)), s2)), rn_mul((T(1) / T(2)), s3)), s4), rn_mul((T(1) / T(2)), s5)), rn_mul((T(1) / T(2)), s6)), rn_mul((T(-1) / T(2)), s10)), rn_mul((T(-1) / T(2)), s11)), rn_mul((T(-1) / T(2)), s17)), rn_mul((T(-1) / T(2)), s18));
  f[19] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(4)), s8), rn_mul((T(-1) / T(4)), s11)), rn_mul((T(-1) / T(4)), s14)), rn_mul((T(1) / T(4)), s17));
  f[20] = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), s2), rn_mul((T(-1) / T(2)), s5)), rn_mul((T(-1) / T(4)), s7)), rn_mul((T(-1) / T(4)), s9)), rn_mul((T(-1) / T(4)), s10)), rn_mul((T(1) / T(4)), s12)), rn_mul((T(1) / T(4)), s13)), rn_mul((T(-1) / T(4)), s15)), rn_mul((T(1) / T(4)), s16)), rn_mul((T(1) / T(4)), s18));
  f[21] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(4)), s9), rn_mul((T(-1) / T(4)), s10)), rn_mul((T(-1) / T(4)), s12)), rn_mul((T(1) / T(4)), s18));
  f[22] = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), s3), rn_mul((T(-1) / T(2)), s6)), rn_mul((T(-1) / T(4)), s7)), rn_mul((T(-1) / T(4)), s8)), rn_mul((T(-1) / T(4)), s11)), rn_mul((T(-1) / T(4)), s13)), rn_mul((T(1) / T(4)), s14)), rn_mul((T(1) / T(4)), s15)), rn_mul((T(1) / T(4)), s16)), rn_mul((T(1) / T(4)), s17));
  f[23] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(4)), s7), rn_mul((T(-1) / T(4)), s13)), rn_mul((T(-1) / T(4)), s15)), rn_mul((T(1) / T(4)), s16));
  f[24] = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), s1), rn_mul((T(-1) / T(2)), s4)), rn_mul((T(-1) / T(4)), s8)), rn_mul((T(-1) / T(4)), s9)), rn_mul((T(1) / T(4)), s10)), rn_mul((T(1) / T(4)), s11)), rn_mul((T(-1) / T(4)), s12)), rn_mul((T(-1) / T(4)), s14)), rn_mul((T(1) / T(4)), s17)), rn_mul((T(1) / T(4)), s18));
  f[26] = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(s0, rn_mul((T(-1) / T(2)), s1)), rn_mul((T(-1) / T(2)), s2)), rn_mul((T(-1) / T(2)), s3)), rn_mul((T(-1) / T(2)), s4)), rn_mul((T(-1) / T(2)), s5)), rn_mul((T(-1) / T(2)), s6)), rn_mul((T(1) / T(4)), s7)), rn_mul((T(1) / T(4)), s8)), rn_mul((T(1) / T(4)), s9)), rn_mul((T(1) / T(4)), s10)), rn_mul((T(1) / T(4)), s11)), rn_mul((T(1) / T(4)), s12)), rn_mul((T(1) / T(4)), s13)), rn_mul((T(1) / T(4)), s14)), rn_mul((T(1) / T(4)), s15)), rn_mul((T(1) / T(4)), s16)), rn_mul((T(1) / T(4)), s17)), rn_mul((T(1) / T(4)), s18));
}
template <typename T>
PSL_HDI void restore_rho_u_n0(const T (&f)[27], T& rho, T& ux, T& uy, T& uz) {
  const T q0 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_mul((T(5) / T(2)), f[0]), rn_mul(T(2), f[2])), rn_mul(T(2), f[3])), rn_mul(T(2), f[5])), rn_mul(T(-2), f[10])), rn_mul(T(-2), f[11])), rn_mul(T(-2), f[18])), rn_mul(T(-16), f[25]));
  const T q1 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), f[0]), rn_mul(T(-2), f[2])), f[3]), f[5]), rn_mul(T(-4), f[10])), rn_mul(T(-4), f[11])), rn_mul(T(2), f[18])), rn_mul(T(-8), f[25]));
  const T q2 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), f[0]), f[2]), f[3]), rn_mul(T(-2), f[5])), rn_mul(T(2), f[10])), rn_mul(T(-4), f[11])), rn_mul(T(-4), f[18])), rn_mul(T(-8), f[25]));
  const T q3 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), f[0]), f[2]), rn_mul(T(-2), f[3])), f[5]), rn_mul(T(-4), f[10])), rn_mul(T(2), f[11])), rn_mul(T(-4), f[18])), rn_mul(T(-8), f[25]));
  rho = q0;
  ux = rn_div(q1, rho);
  uy = rn_div(q2, rho);
  uz = rn_div(q3, rho);
}
template <typename T>
PSL_HDI void restore_u_n0(const T (&f)[27], const T rho, T& ux, T& uy, T& uz) {
  const T scmf0 = rn_div(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add((-f[0]), rn_mul(T(-2), f[2])), rn_mul(T(-2), f[3])), rn_mul(T(-2), f[5])), rn_mul(T(-4), f[10])), rn_mul(T(-4), f[11])), rn_mul(T(-4), f[18])), rn_mul(T(-8), f[25])), rho);
  const T scmf1 = rn_div(rn_add(rn_add(rn_add((-f[0]), rn_mul(T(-2), f[3])), rn_mul(T(-2), f[5])), rn_mul(T(-4), f[18])), rho);
  const T scmf2 = rn_div(rn_add(rn_add(rn_add((-f[0]), rn_mul(T(-2), f[2])), rn_mul(T(-2), f[3])), rn_mul(T(-4), f[10])), rho);
  const T s0 = rn_sub(scmf0, T(-1));
  const T s1 = rn_sub(scmf1, (T(-2) / T(3)));
  const T s2 = rn_sub(scmf2, (T(-2) / T(3)));
  ux = rn_add(s0, rn_mul((T(-3) / T(2)), s1));
  uy = rn_add(s0, rn_mul((T(-3) / T(2)), s2));
  uz = rn_add(rn_add((-s0), rn_mul((T(3) / T(2)), s1)), rn_mul((T(3) / T(2)), s2));
}
template <typename T>
PSL_HDI void restore_rho_n0(const T (&f)[27], T& rho, const T ux, const T uy, const T uz) {
  const T scqu = rn_add(rn_add(rn_mul(T(1), ux), rn_mul(T(1), uy)), rn_mul(T(1), uz));
  const T s = rn_add(T(-1), scqu);
  const T scmf = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add((-f[0]), rn_mul(T(-2), f[2])), rn_mul(T(-2), f[3])), rn_mul(T(-2), f[5])), rn_mul(T(-4), f[10])), rn_mul(T(-4), f[11])), rn_mul(T(-4), f[18])), rn_mul(T(-8), f[25]));
  rho = rn_div(scmf, s);
}
template <typename T>
PSL_HDI void mirror_n0(T (&f)[27]) {
  f[1] = f[2];
  f[4] = f[3];
  f[6] = f[5];
  f[7] = f[10];
  f[8] = f[10];
  f[9] = f[10];
  f[12] = f[11];
  f[13] = f[18];
  f[14] = f[18];
  f[15] = f[11];
  f[16] = f[11];
  f[17] = f[18];
  f[19] = f[25];
  f[20] = f[25];
  f[21] = f[25];
  f[22] = f[25];
  f[23] = f[25];
  f[24] = f[25];
  f[26] = f[25];
}

// ---- outer normal (-1,+1,+1): 19 unknown populations ----
template <typename T>
PSL_HDI void mbbc_n8(T (&f)[27], const T rho, const T ux, const T uy, const T uz) {
  const T smf0 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(f[0], f[2]), f[4]), f[6]), f[8]), f[15]), f[17]), f[24]);
  const T smf1 = rn_sub(rn_sub(rn_sub((-f[2]), f[8]), f[15]), f[24]);
  const T smf2 = rn_add(rn_add(rn_add(f[6], f[15]), f[17]), f[24]);
  const T smf3 = rn_add(rn_add(rn_add(f[4], f[8]), f[17]), f[24]);
  const T smf4 = rn_add(rn_add(rn_add(f[2], f[8]), f[15]), f[24]);
  const T smf5 = rn_add(rn_add(rn_add(f[6], f[15]), f[17]), f[24]);
  const T smf6 = rn_add(rn_add(rn_add(f[4], f[8]), f[17]), f[24]);
  const T smf7 = rn_add(f[17], f[24]);
  const T smf8 = rn_sub((-f[8]), f[24]);
  const T smf9 = rn_sub((-f[15]), f[24]);
  const T smf10 = rn_add(f[15], f[24]);
  const T smf11 = rn_add(f[8], f[24]);
  const T smf12 = rn_sub((-f[15]), f[24]);
  const T smf13 = rn_add(f[17], f[24]);
  const T smf14 = rn_sub((-f[8]), f[24]);
  const T smf15 = rn_add(f[17], f[24]);
  const T smf16 = rn_add(f[17], f[24]);
  const T smf17 = rn_add(f[8], f[24]);
  const T smf18 = rn_add(f[15], f[24]);
  const T m0 = rho;
  const T m1 = rn_mul(rho, ux);
  const T m2 = rn_mul(rho, uy);
  const T m3 = rn_mul(rho, uz);
  const T m4 = rn_add(rn_mul((T(1) / T(3)), rho), rn_mul(rn_mul(rho, ux), ux));
  const T m5 = rn_add(rn_mul((T(1) / T(3)), rho), rn_mul(rn_mul(rho, uy), uy));
  const T m6 = rn_add(rn_mul((T(1) / T(3)), rho), rn_mul(rn_mul(rho, uz), uz));
  const T m7 = rn_mul(rn_mul(rho, uy), uz);
  const T m8 = rn_mul(rn_mul(rho, ux), uz);
  const T m9 = rn_mul(rn_mul(rho, ux), uy);
  const T m10 = rn_add(rn_mul(rn_mul((T(1) / T(3)), rho), uy), rn_mul(rn_mul(rn_mul(rho, ux), ux), uy));
  const T m11 = rn_add(rn_mul(rn_mul((T(1) / T(3)), rho), uz), rn_mul(rn_mul(rn_mul(rho, ux), ux), uz));
  const T m12 = rn_add(rn_mul(rn_mul((T(1) / T(3)), rho), ux), rn_mul(rn_mul(rn_mul(rho, ux), uy), uy));
  const T m13 = rn_add(rn_mul(rn_mul((T(1) / T(3)), rho), uz), rn_mul(rn_mul(rn_mul(rho, uy), uy), uz));
  const T m14 = rn_add(rn_mul(rn_mul((T(1) / T(3)), rho), ux), rn_mul(rn_mul(rn_mul(rho, ux), uz), uz));
  const T m15 = rn_add(rn_mul(rn_mul((T(1) / T(3)), rho), uy), rn_mul(rn_mul(rn_mul(rho, uy), uz), uz));
  const T m16 = rn_add(rn_add(rn_add(rn_mul((T(1) / T(9)), rho), rn_mul(rn_mul(rn_mul((T(1) / T(3)), rho), uy), uy)), rn_mul(rn_mul(rn_mul((T(1) / T(3)), rho), uz), uz)), rn_mul(rn_mul(rn_mul(rn_mul(rho, uy), uy), uz), uz));
  const T m17 = rn_add(rn_add(rn_add(rn_mul((T(1) / T(9)), rho), rn_mul(rn_mul(rn_mul((T(1) / T(3)), rho), ux), ux)), rn_mul(rn_mul(rn_mul((T(1) / T(3)), rho), uz), uz)), rn_mul(rn_mul(rn_mul(rn_mul(rho, ux), ux), uz), uz));
  const T m18 = rn_add(rn_add(rn_add(rn_mul((T(1) / T(9)), rho), rn_mul(rn_mul(rn_mul((T(1) / T(3)), rho), ux), ux)), rn_mul(rn_mul(rn_mul((T(1) / T(3)), rho), uy), uy)), rn_mul(rn_mul(rn_mul(rn_mul(rho, ux), ux), uy), uy));
  const T s0 = rn_sub(m0, smf0);
  const T s1 = rn_sub(m1, smf1);
  const T s2 = rn_sub(m2, smf2);
  const T s3 = rn_sub(m3, smf3);
  const T s4 = rn_sub(m4, smf4);
  const T s5 = rn_sub(m5, smf5);
  const T s6 = rn_sub(m6, smf6);
  const T s7 = rn_sub(m7, smf7);
  const T s8 = rn_sub(m8, smf8);
  const T s9 = rn_sub(m9, smf9);
  const T s10 = rn_sub(m10, smf10);
  const T s11 = rn_sub(m11, smf11);
  const T s12 = rn_sub(m12, smf12);
  const T s13 = rn_sub(m13, smf13);
  const T s14 = rn_sub(m14, smf14);
  const T s15 = rn_sub(m15, smf15);
  const T s16 = rn_sub(m16, smf16);
  const T s17 = rn_sub(m17, smf17);
  const T s18 = rn_sub(m18, smf18);
  f[1] = rn_add(rn_sub(rn_sub(s0, s5), s6), s16);
  f[3] = rn_add(rn_sub(rn_sub(s0, s4), s5), s18);
  f[5] = rn_add(rn_sub(rn_sub(s0, s4), s6), s17);
  f[7] = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add((-s0), rn_mul((T(1) / T(2)), s1)), rn_mul((T(-1) / T(2)), s3)), rn_mul((T(1) / T(2)), s4)), s5), rn_mul((T(1) / T(2)), s6)), rn_mul((T(-1) / T(2)), s12)), rn_mul((T(1) / T(2)), s13)), rn_mul((T(-1) / T(2)), s16)), rn_mul((T(-1) / T(2)), s18));
  f[9] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), s3), rn_mul((T(1) / T(2)), s6)), rn_mul((T(-1) / T(2)), s13)), rn_mul((T(-1) / T(2)), s16));
  f[10] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(2)), s1), rn_mul((T(1) / T(2)), s4)), rn_mul((T(1) / T(2)), s12)), rn_mul((T(-1) / T(2)), s18));
  f[11] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(2)), s1), rn_mul((T(1) / T(2)), s4)), rn_mul((T(1) / T(2)), s14)), rn_mul((T(-1) / T(2)), s17));
  f[12] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), s2), rn_mul((T(1) / T(2)), s5)), rn_mul((T(-1) / T(2)), s15)), rn_mul((T(-1) / T(2)), s16));
  f[13] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), s2), rn_mul((T(1) / T(2)), s5)), rn_mul((T(-1) / T(2)), s10)), rn_mul((T(-1) / T(2)), s18));
  f[14] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), s3), rn_mul((T(1) / T(2)), s6)), rn_mul((T(-1) / T(2)), s11)), rn_mul((T(-1) / T(2)), s17));
  f[16] = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add((-s0), rn_mul((T(1) / T(2)), s1)), rn_mul((T(-1) / T(2)), s2)), rn_mul((T(1) / T(2)), s4)), rn_mul((T(1) / T(2)), s5)), s6), rn_mul((T(-1) / T(2)), s14)), rn_mul((T(1) / T(2)), s15)), rn_mul((T(-1) / T(2)), s16)), rn_mul((T(-1) / T(2)), s17));
  f[18] = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add((-s0), rn_mul((T(-1) / T(2)), s2)), rn_mul((T(-1) / T(2)), s3)), s4), rn_mul((T(1) / T(2)), s5)), rn_mul((T(1) / T(2)), s6)), rn_mul((T(1) / T(2)), s10)), rn_mul((T(1) / T(2)), s11)), rn_mul((T(-1) / T(2)), s17)), rn_mul((T(-1) / T(2)), s18));
  f[19] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(4)), s9), rn_mul((T(1) / T(4)), s10)), rn_mul((T(-1) / T(4)), s12)), rn_mul((T(1) / T(4)), s18));
  f[20] = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_mul((T(-1) / T(2)), s3), rn_mul((T(-1) / T(2)), s6)), rn_mul((T(-1) / T(4)), s7)), rn_mul((T(1) / T(4)), s8)), rn_mul((T(1) / T(4)), s11)), rn_mul((T(1) / T(4)), s13)), rn_mul((T(1) / T(4)), s14)), rn_mul((T(-1) / T(4)), s15)), rn_mul((T(1) / T(4)), s16)), rn_mul((T(1) / T(4)), s17));
  f[21] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(4)), s8), rn_mul((T(1) / T(4)), s11)), rn_mul((T(-1) / T(4)), s14)), rn_mul((T(1) / T(4)), s17));
  f[22] = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_mul((T(-1) / T(2)), s2), rn_mul((T(-1) / T(2)), s5)), rn_mul((T(-1) / T(4)), s7)), rn_mul((T(1) / T(4)), s9)), rn_mul((T(1) / T(4)), s10)), rn_mul((T(1) / T(4)), s12)), rn_mul((T(-1) / T(4)), s13)), rn_mul((T(1) / T(4)), s15)), rn_mul((T(1) / T(4)), s16)), rn_mul((T(1) / T(4)), s18));
  f[23] = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(s0, rn_mul((T(-1) / T(2)), s1)), rn_mul((T(1) / T(2)), s2)), rn_mul((T(1) / T(2)), s3)), rn_mul((T(-1) / T(2)), s4)), rn_mul((T(-1) / T(2)), s5)), rn_mul((T(-1) / T(2)), s6)), rn_mul((T(1) / T(4)), s7)), rn_mul((T(-1) / T(4)), s8)), rn_mul((T(-1) / T(4)), s9)), rn_mul((T(-1) / T(4)), s10)), rn_mul((T(-1) / T(4)), s11)), rn_mul((T(1) / T(4)), s12)), rn_mul((T(-1) / T(4)), s13)), rn_mul((T(1) / T(4)), s14)), rn_mul((T(-1) / T(4)), s15)), rn_mul((T(1) / T(4)), s16)), rn_mul((T(1) / T(4)), s17)), rn_mul((T(1) / T(4)), s18));
  f[25] = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), s1), rn_mul((T(-1) / T(2)), s4)), rn_mul((T(1) / T(4)), s8)), rn_mul((T(1) / T(4)), s9)), rn_mul((T(-1) / T(4)), s10)), rn_mul((T(-1) / T(4)), s11)), rn_mul((T(-1) / T(4)), s12)), rn_mul((T(-1) / T(4)), s14)), rn_mul((T(1) / T(4)), s17)), rn_mul((T(1) / T(4)), s18));
  f[26] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(4)), s7), rn_mul((T(1) / T(4)), s13)), rn_mul((T(1) / T(4)), s15)), rn_mul((T(1) / T(4)), s16));
}
template <typename T>
PSL_HDI void restore_rho_u_n8(const T (&f)[27], T& rho, T& ux, T& uy, T& uz) {
  const T q0 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_mul((T(5) / T(2)), f[0]), rn_mul(T(2), f[2])), rn_mul(T(2), f[4])), rn_mul(T(2), f[6])), rn_mul(T(-2), f[8])), rn_mul(T(-2), f[15])), rn_mul(T(-2), f[17])), rn_mul(T(-16), f[24]));
  const T q1 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), f[0]), rn_mul(T(-2), f[2])), f[4]), f[6]), rn_mul(T(-4), f[8])), rn_mul(T(-4), f[15])), rn_mul(T(2), f[17])), rn_mul(T(-8), f[24]));
  const T q2 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_sub(rn_sub(rn_mul((T(-1) / T(2)), f[0]), f[2]), f[4]), rn_mul(T(2), f[6])), rn_mul(T(-2), f[8])), rn_mul(T(4), f[15])), rn_mul(T(4), f[17])), rn_mul(T(8), f[24]));
  const T q3 = rn_add(rn_add(rn_add(rn_add(rn_sub(rn_add(rn_sub(rn_mul((T(-1) / T(2)), f[0]), f[2]), rn_mul(T(2), f[4])), f[6]), rn_mul(T(4), f[8])), rn_mul(T(-2), f[15])), rn_mul(T(4), f[17])), rn_mul(T(8), f[24]));
  rho = q0;
  ux = rn_div(q1, rho);
  uy = rn_div(q2, rho);
  uz = rn_div(q3, rho);
}
template <typename T>
PSL_HDI void restore_u_n8(const T (&f)[27], const T rho, T& ux, T& uy, T& uz) {
  const T scmf0 = rn_div(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add((-f[0]), rn_mul(T(-2), f[2])), rn_mul(T(-2), f[4])), rn_mul(T(-2), f[6])), rn_mul(T(-4), f[8])), rn_mul(T(-4), f[15])), rn_mul(T(-4), f[17])), rn_mul(T(-8), f[24])), rho);
  const T scmf1 = rn_div(rn_add(rn_add(rn_add((-f[0]), rn_mul(T(-2), f[4])), rn_mul(T(-2), f[6])), rn_mul(T(-4), f[17])), rho);
  const T scmf2 = rn_div(rn_add(rn_add(rn_add(f[0], rn_mul(T(2), f[2])), rn_mul(T(2), f[4])), rn_mul(T(4), f[8])), rho);
  const T s0 = rn_sub(scmf0, T(-1));
  const T s1 = rn_sub(scmf1, (T(-2) / T(3)));
  const T s2 = rn_sub(scmf2, (T(2) / T(3)));
  ux = rn_add(s0, rn_mul((T(-3) / T(2)), s1));
  uy = rn_add((-s0), rn_mul((T(-3) / T(2)), s2));
  uz = rn_add(rn_add(s0, rn_mul((T(-3) / T(2)), s1)), rn_mul((T(3) / T(2)), s2));
}
template <typename T>
PSL_HDI void restore_rho_n8(const T (&f)[27], T& rho, const T ux, const T uy, const T uz) {
  const T scqu = rn_add(rn_add(rn_mul(T(1), ux), rn_mul(T(-1), uy)), rn_mul(T(-1), uz));
  const T s = rn_add(T(-1), scqu);
  const T scmf = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add((-f[0]), rn_mul(T(-2), f[2])), rn_mul(T(-2), f[4])), rn_mul(T(-2), f[6])), rn_mul(T(-4), f[8])), rn_mul(T(-4), f[15])), rn_mul(T(-4), f[17])), rn_mul(T(-8), f[24]));
  rho = rn_div(scmf, s);
}
template <typename T>
PSL_HDI void mirror_n8(T (&f)[27]) {
  f[1] = f[2];
  f[3] = f[4];
  f[5] = f[6];
  f[7] = f[8];
  f[9] = f[8];
  f[10] = f[8];
  f[11] = f[15];
  f[12] = f[15];
  f[13] = f[17];
  f[14] = f[17];
  f[16] = f[15];
  f[18] = f[17];
  f[19] = f[24];
  f[20] = f[24];
  f[21] = f[24];
  f[22] = f[24];
  f[23] = f[24];
  f[25] = f[24];
  f[26] = f[24];
}

// ---- outer normal (+1,-1,+1): 19 unknown populations ----
template <typename T>
PSL_HDI void mbbc_n20(T (&f)[27], const T rho, const T ux, const T uy, const T uz) {
  const T smf0 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(f[0], f[1]), f[4]), f[5]), f[9]), f[14]), f[16]), f[20]);
  const T smf1 = rn_add(rn_add(rn_add(f[1], f[9]), f[16]), f[20]);
  const T smf2 = rn_sub(rn_sub(rn_sub((-f[5]), f[14]), f[16]), f[20]);
  const T smf3 = rn_add(rn_add(rn_add(f[4], f[9]), f[14]), f[20]);
  const T smf4 = rn_add(rn_add(rn_add(f[1], f[9]), f[16]), f[20]);
  const T smf5 = rn_add(rn_add(rn_add(f[5], f[14]), f[16]), f[20]);
  const T smf6 = rn_add(rn_add(rn_add(f[4], f[9]), f[14]), f[20]);
  const T smf7 = rn_sub((-f[14]), f[20]);
  const T smf8 = rn_add(f[9], f[20]);
  const T smf9 = rn_sub((-f[16]), f[20]);
  const T smf10 = rn_sub((-f[16]), f[20]);
  const T smf11 = rn_add(f[9], f[20]);
  const T smf12 = rn_add(f[16], f[20]);
  const T smf13 = rn_add(f[14], f[20]);
  const T smf14 = rn_add(f[9], f[20]);
  const T smf15 = rn_sub((-f[14]), f[20]);
  const T smf16 = rn_add(f[14], f[20]);
  const T smf17 = rn_add(f[9], f[20]);
  const T smf18 = rn_add(f[16], f[20]);
  const T m0 = rho;
  const T m1 = rn_mul(rho, ux);
  const T m2 = rn_mul(rho, uy);
  const T m3 = rn_mul(rho, uz);
  const T m4 = rn_add(rn_mul((T(1) / T(3)), rho), rn_mul(rn_mul(rho, ux), ux));
  const T m5 = rn_add(rn_mul((T(1) / T(3)), rho), rn_mul(rn_mul(rho, uy), uy));
  const T m6 = rn_add(rn_mul((T(1) / T(3)), rho), rn_mul(rn_mul(rho, uz), uz));
  const T m7 = rn_mul(rn_mul(rho, uy), uz);
  const T m8 = rn_mul(rn_mul(rho, ux), uz);
  const T m9 = rn_mul(rn_mul(rho, ux), uy);
  const T m10 = rn_add(rn_mul(rn_mul((T(1) / T(3)), rho), uy), rn_mul(rn_mul(rn_mul(rho, ux), ux), uy));
  const T m11 = rn_add(rn_mul(rn_mul((T(1) / T(3)), rho), uz), rn_mul(rn_mul(rn_mul(rho, ux), ux), uz));
  const T m12 = rn_add(rn_mul(rn_mul((T(1) / T(3)), rho), ux), rn_mul(rn_mul(rn_mul(rho, ux), uy), uy));
  const T m13 = rn_add(rn_mul(rn_mul((T(1) / T(3)), rho), uz), rn_mul(rn_mul(rn_mul(rho, uy), uy), uz));
  const T m14 = rn_add(rn_mul(rn_mul((T(1) / T(3)), rho), ux), rn_mul(rn_mul(rn_mul(rho, ux), uz), uz));
  const T m15 = rn_add(rn_mul(rn_mul((T(1) / T(3)), rho), uy), rn_mul(rn_mul(rn_mul(rho, uy), uz), uz));
  const T m16 = rn_add(rn_add(rn_add(rn_mul((T(1) / T(9)), rho), rn_mul(rn_mul(rn_mul((T(1) / T(3)), rho), uy), uy)), rn_mul(rn_mul(rn_mul((T(1) / T(3)), rho), uz), uz)), rn_mul(rn_mul(rn_mul(rn_mul(rho, uy), uy), uz), uz));
  const T m17 = rn_add(rn_add(rn_add(rn_mul((T(1) / T(9)), rho), rn_mul(rn_mul(rn_mul((T(1) / T(3)), rho), ux), ux)), rn_mul(rn_mul(rn_mul((T(1) / T(3)), rho), uz), uz)), rn_mul(rn_mul(rn_mul(rn_mul(rho, ux), ux), uz), uz));
  const T m18 = rn_add(rn_add(rn_add(rn_mul((T(1) / T(9)), rho), rn_mul(rn_mul(rn_mul((T(1) / T(3)), rho), ux), ux)), rn_mul(rn_mul(rn_mul((T(1) / T(3)), rho), uy), uy)), rn_mul(rn_mul(rn_mul(rn_mul(rho, ux), ux), uy), uy));
  const T s0 = rn_sub(m0, smf0);
  const T s1 = rn_sub(m1, smf1);
  const T s2 = rn_sub(m2, smf2);
  const T s3 = rn_sub(m3, smf3);
  const T s4 = rn_sub(m4, smf4);
  const T s5 = rn_sub(m5, smf5);
  const T s6 = rn_sub(m6, smf6);
  const T s7 = rn_sub(m7, smf7);
  const T s8 = rn_sub(m8, smf8);
  const T s9 = rn_sub(m9, smf9);
  const T s10 = rn_sub(m10, smf10);
  const T s11 = rn_sub(m11, smf11);
  const T s12 = rn_sub(m12, smf12);
  const T s13 = rn_sub(m13, smf13);
  const T s14 = rn_sub(m14, smf14);
  const T s15 = rn_sub(m15, smf15);
  const T s16 = rn_sub(m16, smf16);
  const T s17 = rn_sub(m17, smf17);
  const T s18 = rn_sub(m18, smf18);
  f[2] = rn_add(rn_sub(rn_sub(s0, s5), s6), s16);
  f[3] = rn_add(rn_sub(rn_sub(s0, s4), s5), s18);
  f[6] = rn_add(rn_sub(rn_sub(s0, s4), s6), s17);
  f[7] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), s1), rn_mul((T(1) / T(2)), s4)), rn_mul((T(-1) / T(2)), s12)), rn_mul((T(-1) / T(2)), s18));
  f[8] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), s3), rn_mul((T(1) / T(2)), s6)), rn_mul((T(-1) / T(2)), s13)), rn_mul((T(-1) / T(2)), s16));
  f[10] = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add((-s0), rn_mul((T(-1) / T(2)), s1)), rn_mul((T(-1) / T(2)), s3)), rn_mul((T(1) / T(2)), s4)), s5), rn_mul((T(1) / T(2)), s6)), rn_mul((T(1) / T(2)), s12)), rn_mul((T(1) / T(2)), s13)), rn_mul((T(-1) / T(2)), s16)), rn_mul((T(-1) / T(2)), s18));
  f[11] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(2)), s2), rn_mul((T(1) / T(2)), s5)), rn_mul((T(1) / T(2)), s15)), rn_mul((T(-1) / T(2)), s16));
  f[12] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), s1), rn_mul((T(1) / T(2)), s4)), rn_mul((T(-1) / T(2)), s14)), rn_mul((T(-1) / T(2)), s17));
  f[13] = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add((-s0), rn_mul((T(1) / T(2)), s2)), rn_mul((T(-1) / T(2)), s3)), s4), rn_mul((T(1) / T(2)), s5)), rn_mul((T(1) / T(2)), s6)), rn_mul((T(-1) / T(2)), s10)), rn_mul((T(1) / T(2)), s11)), rn_mul((T(-1) / T(2)), s17)), rn_mul((T(-1) / T(2)), s18));
  f[15] = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add((-s0), rn_mul((T(-1) / T(2)), s1)), rn_mul((T(1) / T(2)), s2)), rn_mul((T(1) / T(2)), s4)), rn_mul((T(1) / T(2)), s5)), s6), rn_mul((T(1) / T(2)), s14)), rn_mul((T(-1) / T(2)), s15)), rn_mul((T(-1) / T(2)), s16)), rn_mul((T(-1) / T(2)), s17));
  f[17] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), s3), rn_mul((T(1) / T(2)), s6)), rn_mul((T(-1) / T(2)), s11)), rn_mul((T(-1) / T(2)), s17));
  f[18] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(2)), s2), rn_mul((T(1) / T(2)), s5)), rn_mul((T(1) / T(2)), s10)), rn_mul((T(-1) / T(2)), s18));
  f[19] = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(s0, rn_mul((T(1) / T(2)), s1)), rn_mul((T(-1) / T(2)), s2)), rn_mul((T(1) / T(2)), s3)), rn_mul((T(-1) / T(2)), s4)), rn_mul((T(-1) / T(2)), s5)), rn_mul((T(-1) / T(2)), s6)), rn_mul((T(-1) / T(4)), s7)), rn_mul((T(1) / T(4)), s8)), rn_mul((T(-1) / T(4)), s9)), rn_mul((T(1) / T(4)), s10)), rn_mul((T(-1) / T(4)), s11)), rn_mul((T(-1) / T(4)), s12)), rn_mul((T(-1) / T(4)), s13)), rn_mul((T(-1) / T(4)), s14)), rn_mul((T(1) / T(4)), s15)), rn_mul((T(1) / T(4)), s16)), rn_mul((T(1) / T(4)), s17)), rn_mul((T(1) / T(4)), s18));
  f[21] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(4)), s7), rn_mul((T(1) / T(4)), s13)), rn_mul((T(-1) / T(4)), s15)), rn_mul((T(1) / T(4)), s16));
  f[22] = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_mul((T(-1) / T(2)), s1), rn_mul((T(-1) / T(2)), s4)), rn_mul((T(-1) / T(4)), s8)), rn_mul((T(1) / T(4)), s9)), rn_mul((T(1) / T(4)), s10)), rn_mul((T(-1) / T(4)), s11)), rn_mul((T(1) / T(4)), s12)), rn_mul((T(1) / T(4)), s14)), rn_mul((T(1) / T(4)), s17)), rn_mul((T(1) / T(4)), s18));
  f[23] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(4)), s9), rn_mul((T(-1) / T(4)), s10)), rn_mul((T(1) / T(4)), s12)), rn_mul((T(1) / T(4)), s18));
  f[24] = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_mul((T(-1) / T(2)), s3), rn_mul((T(-1) / T(2)), s6)), rn_mul((T(1) / T(4)), s7)), rn_mul((T(-1) / T(4)), s8)), rn_mul((T(1) / T(4)), s11)), rn_mul((T(1) / T(4)), s13)), rn_mul((T(-1) / T(4)), s14)), rn_mul((T(1) / T(4)), s15)), rn_mul((T(1) / T(4)), s16)), rn_mul((T(1) / T(4)), s17));
  f[25] = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), s2), rn_mul((T(-1) / T(2)), s5)), rn_mul((T(1) / T(4)), s7)), rn_mul((T(1) / T(4)), s9)), rn_mul((T(-1) / T(4)), s10)), rn_mul((T(-1) / T(4)), s12)), rn_mul((T(-1) / T(4)), s13)), rn_mul((T(-1) / T(4)), s15)), rn_mul((T(1) / T(4)), s16)), rn_mul((T(1) / T(4)), s18));
  f[26] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(4)), s8), rn_mul((T(1) / T(4)), s11)), rn_mul((T(1) / T(4)), s14)), rn_mul((T(1) / T(4)), s17));
}
template <typename T>
PSL_HDI void restore_rho_u_n20(const T (&f)[27], T& rho, T& ux, T& uy, T& uz) {
  const T q0 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_mul((T(5) / T(2)), f[0]), rn_mul(T(2), f[1])), rn_mul(T(2), f[4])), rn_mul(T(2), f[5])), rn_mul(T(-2), f[9])), rn_mul(T(-2), f[14])), rn_mul(T(-2), f[16])), rn_mul(T(-16), f[20]));
  const T q1 = rn_add(rn_add(rn_add(rn_add(rn_sub(rn_sub(rn_add(rn_mul((T(-1) / T(2)), f[0]), rn_mul(T(2), f[1])), f[4]), f[5]), rn_mul(T(4), f[9])), rn_mul(T(-2), f[14])), rn_mul(T(4), f[16])), rn_mul(T(8), f[20]));
  const T q2 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), f[0]), f[1]), f[4]), rn_mul(T(-2), f[5])), rn_mul(T(2), f[9])), rn_mul(T(-4), f[14])), rn_mul(T(-4), f[16])), rn_mul(T(-8), f[20]));
  const T q3 = rn_add(rn_add(rn_add(rn_add(rn_sub(rn_add(rn_sub(rn_mul((T(-1) / T(2)), f[0]), f[1]), rn_mul(T(2), f[4])), f[5]), rn_mul(T(4), f[9])), rn_mul(T(4), f[14])), rn_mul(T(-2), f[16])), rn_mul(T(8), f[20]));
  rho = q0;
  ux = rn_div(q1, rho);
  uy = rn_div(q2, rho);
  uz = rn_div(q3, rho);
}
template <typename T>
PSL_HDI void restore_u_n20(const T (&f)[27], const T rho, T& ux, T& uy, T& uz) {
  const T scmf0 = rn_div(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add((-f[0]), rn_mul(T(-2), f[1])), rn_mul(T(-2), f[4])), rn_mul(T(-2), f[5])), rn_mul(T(-4), f[9])), rn_mul(T(-4), f[14])), rn_mul(T(-4), f[16])), rn_mul(T(-8), f[20])), rho);
  const T scmf1 = rn_div(rn_add(rn_add(rn_add(f[0], rn_mul(T(2), f[4])), rn_mul(T(2), f[5])), rn_mul(T(4), f[14])), rho);
  const T scmf2 = rn_div(rn_add(rn_add(rn_add((-f[0]), rn_mul(T(-2), f[1])), rn_mul(T(-2), f[4])), rn_mul(T(-4), f[9])), rho);
  const T s0 = rn_sub(scmf0, T(-1));
  const T s1 = rn_sub(scmf1, (T(2) / T(3)));
  const T s2 = rn_sub(scmf2, (T(-2) / T(3)));
  ux = rn_add((-s0), rn_mul((T(-3) / T(2)), s1));
  uy = rn_add(s0, rn_mul((T(-3) / T(2)), s2));
  uz = rn_add(rn_add(s0, rn_mul((T(3) / T(2)), s1)), rn_mul((T(-3) / T(2)), s2));
}
template <typename T>
PSL_HDI void restore_rho_n20(const T (&f)[27], T& rho, const T ux, const T uy, const T uz) {
  const T scqu = rn_add(rn_add(rn_mul(T(-1), ux), rn_mul(T(1), uy)), rn_mul(T(-1), uz));
  const T s = rn_add(T(-1), scqu);
  const T scmf = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add((-f[0]), rn_mul(T(-2), f[1])), rn_mul(T(-2), f[4])), rn_mul(T(-2), f[5])), rn_mul(T(-4), f[9])), rn_mul(T(-4), f[14])), rn_mul(T(-4), f[16])), rn_mul(T(-8), f[20]));
  rho = rn_div(scmf, s);
}
template <typename T>
PSL_HDI void mirror_n20(T (&f)[27]) {
  f[2] = f[1];
  f[3] = f[4];
  f[6] = f[5];
  f[7] = f[9];
  f[8] = f[9];
  f[10] = f[9];
  f[11] = f[16];
  f[12] = f[16];
  f[13] = f[14];
  f[15] = f[16];
  f[17] = f[14];
  f[18] = f[14];
  f[19] = f[20];
  f[21] = f[20];
  f[22] = f[20];
  f[23] = f[20];
  f[24] = f[20];
  f[25] = f[20];
  f[26] = f[20];
}

// ---- outer normal (+1,+1,-1): 19 unknown populations ----
template <typename T>
PSL_HDI void mbbc_n24(T (&f)[27], const T rho, const T ux, const T uy, const T uz) {
  const T smf0 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(f[0], f[1]), f[3]), f[6]), f[7]), f[12]), f[13]), f[22]);
  const T smf1 = rn_add(rn_add(rn_add(f[1], f[7]), f[12]), f[22]);
  const T smf2 = rn_add(rn_add(rn_add(f[6], f[12]), f[13]), f[22]);
  const T smf3 = rn_sub(rn_sub(rn_sub((-f[3]), f[7]), f[13]), f[22]);
  const T smf4 = rn_add(rn_add(rn_add(f[1], f[7]), f[12]), f[22]);
  const T smf5 = rn_add(rn_add(rn_add(f[6], f[12]), f[13]), f[22]);
  const T smf6 = rn_add(rn_add(rn_add(f[3], f[7]), f[13]), f[22]);
  const T smf7 = rn_sub((-f[13]), f[22]);
  const T smf8 = rn_sub((-f[7]), f[22]);
  const T smf9 = rn_add(f[12], f[22]);
  const T smf10 = rn_add(f[12], f[22]);
  const T smf11 = rn_sub((-f[7]), f[22]);
  const T smf12 = rn_add(f[12], f[22]);
  const T smf13 = rn_sub((-f[13]), f[22]);
  const T smf14 = rn_add(f[7], f[22]);
  const T smf15 = rn_add(f[13], f[22]);
  const T smf16 = rn_add(f[13], f[22]);
  const T smf17 = rn_add(f[7], f[22]);
  const T smf18 = rn_add(f[12], f[22]);
  const T m0 = rho;
  const T m1 = rn_mul(rho, ux);
  const T m2 = rn_mul(rho, uy);
  const T m3 = rn_mul(rho, uz);
  const T m4 = rn_add(rn_mul((T(1) / T(3)), rho), rn_mul(rn_mul(rho, ux), ux));
  const T m5 = rn_add(rn_mul((T(1) / T(3)), rho), rn_mul(rn_mul(rho, uy), uy));
  const T m6 = rn_add(rn_mul((T(1) / T(3)), rho), rn_mul(rn_mul(rho, uz), uz));
  const T m7 = rn_mul(rn_mul(rho, uy), uz);
  const T m8 = rn_mul(rn_mul(rho, ux), uz);
  const T m9 = rn_mul(rn_mul(rho, ux), uy);
  const T m10 = rn_add(rn_mul(rn_mul((T(1) / T(3)), rho), uy), rn_mul(rn_mul(rn_mul(rho, ux), ux), uy));
  const T m11 = rn_add(rn_mul(rn_mul((T(1) / T(3)), rho), uz), rn_mul(rn_mul(rn_mul(rho, ux), ux), uz));
  const T m12 = rn_add(rn_mul(rn_mul((T(1) / T(3)), rho), ux), rn_mul(rn_mul(rn_mul(rho, ux), uy), uy));
  const T m13 = rn_add(rn_mul(rn_mul((T(1) / T(3)), rho), uz), rn_mul(rn_mul(rn_mul(rho, uy), uy), uz));
  const T m14 = rn_add(rn_mul(rn_mul((T(1) / T(3)), rho), ux), rn_mul(rn_mul(rn_mul(rho, ux), uz), uz));
  const T m15 = rn_add(rn_mul(rn_mul((T(1) / T(3)), rho), uy), rn_mul(rn_mul(rn_mul(rho, uy), uz), uz));
  const T m16 = rn_add(rn_add(rn_add(rn_mul((T(1) / T(9)), rho), rn_mul(rn_mul(rn_mul((T(1) / T(3)), rho), uy), uy)), rn_mul(rn_mul(rn_mul((T(1) / T(3)), rho), uz), uz)), rn_mul(rn_mul(rn_mul(rn_mul(rho, uy), uy), uz), uz));
  const T m17 = rn_add(rn_add(rn_add(rn_mul((T(1) / T(9)), rho), rn_mul(rn_mul(rn_mul((T(1) / T(3)), rho), ux), ux)), rn_mul(rn_mul(rn_mul((T(1) / T(3)), rho), uz), uz)), rn_mul(rn_mul(rn_mul(rn_mul(rho, ux), ux), uz), uz));
  const T m18 = rn_add(rn_add(rn_add(rn_mul((T(1) / T(9)), rho), rn_mul(rn_mul(rn_mul((T(1) / T(3)), rho), ux), ux)), rn_mul(rn_mul(rn_mul((T(1) / T(3)), rho), uy), uy)), rn_mul(rn_mul(rn_mul(rn_mul(rho, ux), ux), uy), uy));
  const T s0 = rn_sub(m0, smf0);
  const T s1 = rn_sub(m1, smf1);
  const T s2 = rn_sub(m2, smf2);
  const T s3 = rn_sub(m3, smf3);
  const T s4 = rn_sub(m4, smf4);
  const T s5 = rn_sub(m5, smf5);
  const T s6 = rn_sub(m6, smf6);
  const T s7 = rn_sub(m7, smf7);
  const T s8 = rn_sub(m8, smf8);
  const T s9 = rn_sub(m9, smf9);
  const T s10 = rn_sub(m10, smf10);
  const T s11 = rn_sub(m11, smf11);
  const T s12 = rn_sub(m12, smf12);
  const T s13 = rn_sub(m13, smf13);
  const T s14 = rn_sub(m14, smf14);
  const T s15 = rn_sub(m15, smf15);
  const T s16 = rn_sub(m16, smf16);
  const T s17 = rn_sub(m17, smf17);
  const T s18 = rn_sub(m18, smf18);
  f[2] = rn_add(rn_sub(rn_sub(s0, s5), s6), s16);
  f[4] = rn_add(rn_sub(rn_sub(s0, s4), s5), s18);
  f[5] = rn_add(rn_sub(rn_sub(s0, s4), s6), s17);
  f[8] = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add((-s0), rn_mul((T(-1) / T(2)), s1)), rn_mul((T(1) / T(2)), s3)), rn_mul((T(1) / T(2)), s4)), s5), rn_mul((T(1) / T(2)), s6)), rn_mul((T(1) / T(2)), s12)), rn_mul((T(-1) / T(2)), s13)), rn_mul((T(-1) / T(2)), s16)), rn_mul((T(-1) / T(2)), s18));
  f[9] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), s1), rn_mul((T(1) / T(2)), s4)), rn_mul((T(-1) / T(2)), s12)), rn_mul((T(-1) / T(2)), s18));
  f[10] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(2)), s3), rn_mul((T(1) / T(2)), s6)), rn_mul((T(1) / T(2)), s13)), rn_mul((T(-1) / T(2)), s16));
  f[11] = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add((-s0), rn_mul((T(-1) / T(2)), s1)), rn_mul((T(-1) / T(2)), s2)), rn_mul((T(1) / T(2)), s4)), rn_mul((T(1) / T(2)), s5)), s6), rn_mul((T(1) / T(2)), s14)), rn_mul((T(1) / T(2)), s15)), rn_mul((T(-1) / T(2)), s16)), rn_mul((T(-1) / T(2)), s17));
  f[14] = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add((-s0), rn_mul((T(-1) / T(2)), s2)), rn_mul((T(1) / T(2)), s3)), s4), rn_mul((T(1) / T(2)), s5)), rn_mul((T(1) / T(2)), s6)), rn_mul((T(1) / T(2)), s10)), rn_mul((T(-1) / T(2)), s11)), rn_mul((T(-1) / T(2)), s17)), rn_mul((T(-1) / T(2)), s18));
  f[15] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), s2), rn_mul((T(1) / T(2)), s5)), rn_mul((T(-1) / T(2)), s15)), rn_mul((T(-1) / T(2)), s16));
  f[16] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), s1), rn_mul((T(1) / T(2)), s4)), rn_mul((T(-1) / T(2)), s14)), rn_mul((T(-1) / T(2)), s17));
  f[17] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), s2), rn_mul((T(1) / T(2)), s5)), rn_mul((T(-1) / T(2)), s10)), rn_mul((T(-1) / T(2)), s18));
  f[18] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(2)), s3), rn_mul((T(1) / T(2)), s6)), rn_mul((T(1) / T(2)), s11)), rn_mul((T(-1) / T(2)), s17));
  f[19] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(4)), s7), rn_mul((T(-1) / T(4)), s13)), rn_mul((T(1) / T(4)), s15)), rn_mul((T(1) / T(4)), s16));
  f[20] = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_mul((T(-1) / T(2)), s1), rn_mul((T(-1) / T(2)), s4)), rn_mul((T(1) / T(4)), s8)), rn_mul((T(-1) / T(4)), s9)), rn_mul((T(-1) / T(4)), s10)), rn_mul((T(1) / T(4)), s11)), rn_mul((T(1) / T(4)), s12)), rn_mul((T(1) / T(4)), s14)), rn_mul((T(1) / T(4)), s17)), rn_mul((T(1) / T(4)), s18));
  f[21] = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(s0, rn_mul((T(1) / T(2)), s1)), rn_mul((T(1) / T(2)), s2)), rn_mul((T(-1) / T(2)), s3)), rn_mul((T(-1) / T(2)), s4)), rn_mul((T(-1) / T(2)), s5)), rn_mul((T(-1) / T(2)), s6)), rn_mul((T(-1) / T(4)), s7)), rn_mul((T(-1) / T(4)), s8)), rn_mul((T(1) / T(4)), s9)), rn_mul((T(-1) / T(4)), s10)), rn_mul((T(1) / T(4)), s11)), rn_mul((T(-1) / T(4)), s12)), rn_mul((T(1) / T(4)), s13)), rn_mul((T(-1) / T(4)), s14)), rn_mul((T(-1) / T(4)), s15)), rn_mul((T(1) / T(4)), s16)), rn_mul((T(1) / T(4)), s17)), rn_mul((T(1) / T(4)), s18));
  f[23] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(4)), s8), rn_mul((T(-1) / T(4)), s11)), rn_mul((T(1) / T(4)), s14)), rn_mul((T(1) / T(4)), s17));
  f[24] = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_mul((T(-1) / T(2)), s2), rn_mul((T(-1) / T(2)), s5)), rn_mul((T(1) / T(4)), s7)), rn_mul((T(-1) / T(4)), s9)), rn_mul((T(1) / T(4)), s10)), rn_mul((T(-1) / T(4)), s12)), rn_mul((T(1) / T(4)), s13)), rn_mul((T(1) / T(4)), s15)), rn_mul((T(1) / T(4)), s16)), rn_mul((T(1) / T(4)), s18));
  f[25] = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), s3), rn_mul((T(-1) / T(2)), s6)), rn_mul((T(1) / T(4)), s7)), rn_mul((T(1) / T(4)), s8)), rn_mul((T(-1) / T(4)), s11)), rn_mul((T(-1) / T(4)), s13)), rn_mul((T(-1) / T(4)), s14)), rn_mul((T(-1) / T(4)), s15)), rn_mul((T(1) / T(4)), s16)), rn_mul((T(1) / T(4)), s17));
  f[26] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(4)), s9), rn_mul((T(1) / T(4)), s10)), rn_mul((T(1) / T(4)), s12)), rn_mul((T(1) / T(4)), s18));
}
template <typename T>
PSL_HDI void restore_rho_u_n24(const T (&f)[27], T& rho, T& ux, T& uy, T& uz) {
  const T q0 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_mul((T(5) / T(2)), f[0]), rn_mul(T(2), f[1])), rn_mul(T(2), f[3])), rn_mul(T(2), f[6])), rn_mul(T(-2), f[7])), rn_mul(T(-2), f[12])), rn_mul(T(-2), f[13])), rn_mul(T(-16), f[22]));
  const T q1 = rn_add(rn_add(rn_add(rn_add(rn_sub(rn_sub(rn_add(rn_mul((T(-1) / T(2)), f[0]), rn_mul(T(2), f[1])), f[3]), f[6]), rn_mul(T(4), f[7])), rn_mul(T(4), f[12])), rn_mul(T(-2), f[13])), rn_mul(T(8), f[22]));
  const T q2 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_sub(rn_sub(rn_mul((T(-1) / T(2)), f[0]), f[1]), f[3]), rn_mul(T(2), f[6])), rn_mul(T(-2), f[7])), rn_mul(T(4), f[12])), rn_mul(T(4), f[13])), rn_mul(T(8), f[22]));
  const T q3 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), f[0]), f[1]), rn_mul(T(-2), f[3])), f[6]), rn_mul(T(-4), f[7])), rn_mul(T(2), f[12])), rn_mul(T(-4), f[13])), rn_mul(T(-8), f[22]));
  rho = q0;
  ux = rn_div(q1, rho);
  uy = rn_div(q2, rho);
  uz = rn_div(q3, rho);
}
template <typename T>
PSL_HDI void restore_u_n24(const T (&f)[27], const T rho, T& ux, T& uy, T& uz) {
  const T scmf0 = rn_div(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add((-f[0]), rn_mul(T(-2), f[1])), rn_mul(T(-2), f[3])), rn_mul(T(-2), f[6])), rn_mul(T(-4), f[7])), rn_mul(T(-4), f[12])), rn_mul(T(-4), f[13])), rn_mul(T(-8), f[22])), rho);
  const T scmf1 = rn_div(rn_add(rn_add(rn_add(f[0], rn_mul(T(2), f[3])), rn_mul(T(2), f[6])), rn_mul(T(4), f[13])), rho);
  const T scmf2 = rn_div(rn_add(rn_add(rn_add(f[0], rn_mul(T(2), f[1])), rn_mul(T(2), f[3])), rn_mul(T(4), f[7])), rho);
  const T s0 = rn_sub(scmf0, T(-1));
  const T s1 = rn_sub(scmf1, (T(2) / T(3)));
  const T s2 = rn_sub(scmf2, (T(2) / T(3)));
  ux = rn_add((-s0), rn_mul((T(-3) / T(2)), s1));
  uy = rn_add((-s0), rn_mul((T(-3) / T(2)), s2));
  uz = rn_add(rn_add((-s0), rn_mul((T(-3) / T(2)), s1)), rn_mul((T(-3) / T(2)), s2));
}
template <typename T>
PSL_HDI void restore_rho_n24(const T (&f)[27], T& rho, const T ux, const T uy, const T uz) {
  const T scqu = rn_add(rn_add(rn_mul(T(-1), ux), rn_mul(T(-1), uy)), rn_mul(T(1), uz));
  const T s = rn_add(T(-1), scqu);
  const T scmf = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add((-f[0]), rn_mul(T(-2), f[1])), rn_mul(T(-2), f[3])), rn_mul(T(-2), f[6])), rn_mul(T(-4), f[7])), rn_mul(T(-4), f[12])), rn_mul(T(-4), f[13])), rn_mul(T(-8), f[22]));
  rho = rn_div(scmf, s);
}
template <typename T>
PSL_HDI void mirror_n24(T (&f)[27]) {
  f[2] = f[1];
  f[4] = f[3];
  f[5] = f[6];
  f[8] = f[7];
  f[9] = f[7];
  f[10] = f[7];
  f[11] = f[12];
  f[14] = f[13];
  f[15] = f[12];
  f[16] = f[12];
  f[17] = f[13];
  f[18] = f[13];
  f[19] = f[22];
  f[20] = f[22];
  f[21] = f[22];
  f[23] = f[22];
  f[24] = f[22];
  f[25] = f[22];
  f[26] = f[22];
}

// ---- outer normal (+1,-1,-1): 19 unknown populations ----
template <typename T>
PSL_HDI void mbbc_n18(T (&f)[27], const T rho, const T ux, const T uy, const T uz) {
  const T smf0 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(f[0], f[1]), f[3]), f[5]), f[7]), f[16]), f[18]), f[23]);
  const T smf1 = rn_add(rn_add(rn_add(f[1], f[7]), f[16]), f[23]);
  const T smf2 = rn_sub(rn_sub(rn_sub((-f[5]), f[16]), f[18]), f[23]);
  const T smf3 = rn_sub(rn_sub(rn_sub((-f[3]), f[7]), f[18]), f[23]);
  const T smf4 = rn_add(rn_add(rn_add(f[1], f[7]), f[16]), f[23]);
  const T smf5 = rn_add(rn_add(rn_add(f[5], f[16]), f[18]), f[23]);
  const T smf6 = rn_add(rn_add(rn_add(f[3], f[7]), f[18]), f[23]);
  const T smf7 = rn_add(f[18], f[23]);
  const T smf8 = rn_sub((-f[7]), f[23]);
  const T smf9 = rn_sub((-f[16]), f[23]);
  const T smf10 = rn_sub((-f[16]), f[23]);
  const T smf11 = rn_sub((-f[7]), f[23]);
  const T smf12 = rn_add(f[16], f[23]);
  const T smf13 = rn_sub((-f[18]), f[23]);
  const T smf14 = rn_add(f[7], f[23]);
  const T smf15 = rn_sub((-f[18]), f[23]);
  const T smf16 = rn_add(f[18], f[23]);
  const T smf17 = rn_add(f[7], f[23]);
  const T smf18 = rn_add(f[16], f[23]);
  const T m0 = rho;
  const T m1 = rn_mul(rho, ux);
  const T m2 = rn_mul(rho, uy);
  const T m3 = rn_mul(rho, uz);
  const T m4 = rn_add(rn_mul((T(1) / T(3)), rho), rn_mul(rn_mul(rho, ux), ux));
  const T m5 = rn_add(rn_mul((T(1) / T(3)), rho), rn_mul(rn_mul(rho, uy), uy));
  const T m6 = rn_add(rn_mul((T(1) / T(3)), rho), rn_mul(rn_mul(rho, uz), uz));
  const T m7 = rn_mul(rn_mul(rho, uy), uz);
  const T m8 = rn_mul(rn_mul(rho, ux), uz);
  const T m9 = rn_mul(rn_mul(rho, ux), uy);
  const T m10 = rn_add(rn_mul(rn_mul((T(1) / T(3)), rho), uy), rn_mul(rn_mul(rn_mul(rho, ux), ux), uy));
  const T m11 = rn_add(rn_mul(rn_mul((T(1) / T(3)), rho), uz), rn_mul(rn_mul(rn_mul(rho, ux), ux), uz));
  const T m12 = rn_add(rn_mul(rn_mul((T(1) / T(3)), rho), ux), rn_mul(rn_mul(rn_mul(rho, ux), uy), uy));
  const T m13 = rn_add(rn_mul(rn_mul((T(1) / T(3)), rho), uz), rn_mul(rn_mul(rn_mul(rho, uy), uy), uz));
  const T m14 = rn_add(rn_mul(rn_mul((T(1) / T(3)), rho), ux), rn_mul(rn_mul(rn_mul(rho, ux), uz), uz));
  const T m15 = rn_add(rn_mul(rn_mul((T(1) / T(3)), rho), uy), rn_mul(rn_mul(rn_mul(rho, uy), uz), uz));
  const T m16 = rn_add(rn_add(rn_add(rn_mul((T(1) / T(9)), rho), rn_mul(rn_mul(rn_mul((T(1) / T(3)), rho), uy), uy)), rn_mul(rn_mul(rn_mul((T(1) / T(3)), rho), uz), uz)), rn_mul(rn_mul(rn_mul(rn_mul(rho, uy), uy), uz), uz));
  const T m17 = rn_add(rn_add(rn_add(rn_mul((T(1) / T(9)), rho), rn_mul(rn_mul(rn_mul((T(1) / T(3)), rho), ux), ux)), rn_mul(rn_mul(rn_mul((T(1) / T(3)), rho), uz), uz)), rn_mul(rn_mul(rn_mul(rn_mul(rho, ux), ux), uz), uz));
  const T m18 = rn_add(rn_add(rn_add(rn_mul((T(1) / T(9)), rho), rn_mul(rn_mul(rn_mul((T(1) / T(3)), rho), ux), ux)), rn_mul(rn_mul(rn_mul((T(1) / T(3)), rho), uy), uy)), rn_mul(rn_mul(rn_mul(rn_mul(rho, ux), ux), uy), uy));
  const T s0 = rn_sub(m0, smf0);
  const T s1 = rn_sub(m1, smf1);
  const T s2 = rn_sub(m2, smf2);
  const T s3 = rn_sub(m3, smf3);
  const T s4 = rn_sub(m4, smf4);
  const T s5 = rn_sub(m5, smf5);
  const T s6 = rn_sub(m6, smf6);
  const T s7 = rn_sub(m7, smf7);
  const T s8 = rn_sub(m8, smf8);
  const T s9 = rn_sub(m9, smf9);
  const T s10 = rn_sub(m10, smf10);
  const T s11 = rn_sub(m11, smf11);
  const T s12 = rn_sub(m12, smf12);
  const T s13 = rn_sub(m13, smf13);
  const T s14 = rn_sub(m14, smf14);
  const T s15 = rn_sub(m15, smf15);
  const T s16 = rn_sub(m16, smf16);
  const T s17 = rn_sub(m17, smf17);
  const T s18 = rn_sub(m18, smf18);
  f[2] = rn_add(rn_sub(rn_sub(s0, s5), s6), s16);
  f[4] = rn_add(rn_sub(rn_sub(s0, s4), s5), s18);
  f[6] = rn_add(rn_sub(rn_sub(s0, s4), s6), s17);
  f[8] = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add((-s0), rn_mul((T(-1) / T(2)), s1)), rn_mul((T(1) / T(2)), s3)), rn_mul((T(1) / T(2)), s4)), s5), rn_mul((T(1) / T(2)), s6)), rn_mul((T(1) / T(2)), s12)), rn_mul((T(-1) / T(2)), s13)), rn_mul((T(-1) / T(2)), s16)), rn_mul((T(-1) / T(2)), s18));
  f[9] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), s1), rn_mul((T(1) / T(2)), s4)), rn_mul((T(-1) / T(2)), s12)), rn_mul((T(-1) / T(2)), s18));
  f[10] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(2)), s3), rn_mul((T(1) / T(2)), s6)), rn_mul((T(1) / T(2)), s13)), rn_mul((T(-1) / T(2)), s16));
  f[11] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(2)), s2), rn_mul((T(1) / T(2)), s5)), rn_mul((T(1) / T(2)), s15)), rn_mul((T(-1) / T(2)), s16));
  f[12] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), s1), rn_mul((T(1) / T(2)), s4)), rn_mul((T(-1) / T(2)), s14)), rn_mul((T(-1) / T(2)), s17));
  f[13] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(2)), s3), rn_mul((T(1) / T(2)), s6)), rn_mul((T(1) / T(2)), s11)), rn_mul((T(-1) / T(2)), s17));
  f[14] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(2)), s2), rn_mul((T(1) / T(2)), s5)), rn_mul((T(1) / T(2)), s10)), rn_mul((T(-1) / T(2)), s18));
  f[15] = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add((-s0), rn_mul((T(-1) / T(2)), s1)), rn_mul((T(1) / T(2)), s2)), rn_mul((T(1) / T(2)), s4)), rn_mul((T(1) / T(2)), s5)), s6), rn_mul((T(1) / T(2)), s14)), rn_mul((T(-1) / T(2)), s15)), rn_mul((T(-1) / T(2)), s16)), rn_mul((T(-1) / T(2)), s17));
  f[17] = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add((-s0), rn_mul((T(1) / T(2)), s2)), rn_mul((T(1) / T(2)), s3)), s4), rn_mul((T(1) / T(2)), s5)), rn_mul((T(1) / T(2)), s6)), rn_mul((T(-1) / T(2)), s10)), rn_mul((T(-1) / T(2)), s11)), rn_mul((T(-1) / T(2)), s17)), rn_mul((T(-1) / T(2)), s18));
  f[19] = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), s3), rn_mul((T(-1) / T(2)), s6)), rn_mul((T(-1) / T(4)), s7)), rn_mul((T(1) / T(4)), s8)), rn_mul((T(-1) / T(4)), s11)), rn_mul((T(-1) / T(4)), s13)), rn_mul((T(-1) / T(4)), s14)), rn_mul((T(1) / T(4)), s15)), rn_mul((T(1) / T(4)), s16)), rn_mul((T(1) / T(4)), s17));
  f[20] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(4)), s9), rn_mul((T(-1) / T(4)), s10)), rn_mul((T(1) / T(4)), s12)), rn_mul((T(1) / T(4)), s18));
  f[21] = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), s2), rn_mul((T(-1) / T(2)), s5)), rn_mul((T(-1) / T(4)), s7)), rn_mul((T(1) / T(4)), s9)), rn_mul((T(-1) / T(4)), s10)), rn_mul((T(-1) / T(4)), s12)), rn_mul((T(1) / T(4)), s13)), rn_mul((T(-1) / T(4)), s15)), rn_mul((T(1) / T(4)), s16)), rn_mul((T(1) / T(4)), s18));
  f[22] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(4)), s8), rn_mul((T(-1) / T(4)), s11)), rn_mul((T(1) / T(4)), s14)), rn_mul((T(1) / T(4)), s17));
  f[24] = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(s0, rn_mul((T(1) / T(2)), s1)), rn_mul((T(-1) / T(2)), s2)), rn_mul((T(-1) / T(2)), s3)), rn_mul((T(-1) / T(2)), s4)), rn_mul((T(-1) / T(2)), s5)), rn_mul((T(-1) / T(2)), s6)), rn_mul((T(1) / T(4)), s7)), rn_mul((T(-1) / T(4)), s8)), rn_mul((T(-1) / T(4)), s9)), rn_mul((T(1) / T(4)), s10)), rn_mul((T(1) / T(4)), s11)), rn_mul((T(-1) / T(4)), s12)), rn_mul((T(1) / T(4)), s13)), rn_mul((T(-1) / T(4)), s14)), rn_mul((T(1) / T(4)), s15)), rn_mul((T(1) / T(4)), s16)), rn_mul((T(1) / T(4)), s17)), rn_mul((T(1) / T(4)), s18));
  f[25] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(4)), s7), rn_mul((T(-1) / T(4)), s13)), rn_mul((T(-1) / T(4)), s15)), rn_mul((T(1) / T(4)), s16));
  f[26] = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_mul((T(-1) / T(2)), s1), rn_mul((T(-1) / T(2)), s4)), rn_mul((T(1) / T(4)), s8)), rn_mul((T(1) / T(4)), s9)), rn_mul((T(1) / T(4)), s10)), rn_mul((T(1) / T(4)), s11)), rn_mul((T(1) / T(4)), s12)), rn_mul((T(1) / T(4)), s14)), rn_mul((T(1) / T(4)), s17)), rn_mul((T(1) / T(4)), s18));
}
template <typename T>
PSL_HDI void restore_rho_u_n18(const T (&f)[27], T& rho, T& ux, T& uy, T& uz) {
  const T q0 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_mul((T(5) / T(2)), f[0]), rn_mul(T(2), f[1])), rn_mul(T(2), f[3])), rn_mul(T(2), f[5])), rn_mul(T(-2), f[7])), rn_mul(T(-2), f[16])), rn_mul(T(-2), f[18])), rn_mul(T(-16), f[23]));
  const T q1 = rn_add(rn_add(rn_add(rn_add(rn_sub(rn_sub(rn_add(rn_mul((T(-1) / T(2)), f[0]), rn_mul(T(2), f[1])), f[3]), f[5]), rn_mul(T(4), f[7])), rn_mul(T(4), f[16])), rn_mul(T(-2), f[18])), rn_mul(T(8), f[23]));
  const T q2 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), f[0]), f[1]), f[3]), rn_mul(T(-2), f[5])), rn_mul(T(2), f[7])), rn_mul(T(-4), f[16])), rn_mul(T(-4), f[18])), rn_mul(T(-8), f[23]));
  const T q3 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), f[0]), f[1]), rn_mul(T(-2), f[3])), f[5]), rn_mul(T(-4), f[7])), rn_mul(T(2), f[16])), rn_mul(T(-4), f[18])), rn_mul(T(-8), f[23]));
  rho = q0;
  ux = rn_div(q1, rho);
  uy = rn_div(q2, rho);
  uz = rn_div(q3, rho);
}
template <typename T>
PSL_HDI void restore_u_n18(const T (&f)[27], const T rho, T& ux, T& uy, T& uz) {
  const T scmf0 = rn_div(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(f[0], rn_mul(T(2), f[1])), rn_mul(T(2), f[3])), rn_mul(T(2), f[5])), rn_mul(T(4), f[7])), rn_mul(T(4), f[16])), rn_mul(T(4), f[18])), rn_mul(T(8), f[23])), rho);
  const T scmf1 = rn_div(rn_add(rn_add(rn_add((-f[0]), rn_mul(T(-2), f[3])), rn_mul(T(-2), f[5])), rn_mul(T(-4), f[18])), rho);
  const T scmf2 = rn_div(rn_add(rn_add(rn_add(f[0], rn_mul(T(2), f[1])), rn_mul(T(2), f[3])), rn_mul(T(4), f[7])), rho);
  const T s0 = rn_sub(scmf0, T(1));
  const T s1 = rn_sub(scmf1, (T(-2) / T(3)));
  const T s2 = rn_sub(scmf2, (T(2) / T(3)));
  ux = rn_add(s0, rn_mul((T(3) / T(2)), s1));
  uy = rn_add((-s0), rn_mul((T(3) / T(2)), s2));
  uz = rn_add(rn_add(s0, rn_mul((T(3) / T(2)), s1)), rn_mul((T(-3) / T(2)), s2));
}
template <typename T>
PSL_HDI void restore_rho_n18(const T (&f)[27], T& rho, const T ux, const T uy, const T uz) {
  const T scqu = rn_add(rn_add(rn_mul(T(1), ux), rn_mul(T(-1), uy)), rn_mul(T(-1), uz));
  const T s = rn_add(T(1), scqu);
  const T scmf = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(f[0], rn_mul(T(2), f[1])), rn_mul(T(2), f[3])), rn_mul(T(2), f[5])), rn_mul(T(4), f[7])), rn_mul(T(4), f[16])), rn_mul(T(4), f[18])), rn_mul(T(8), f[23]));
  rho = rn_div(scmf, s);
}
template <typename T>
PSL_HDI void mirror_n18(T (&f)[27]) {
  f[2] = f[1];
  f[4] = f[3];
  f[6] = f[5];
  f[8] = f[7];
  f[9] = f[7];
  f[10] = f[7];
  f[11] = f[16];
  f[12] = f[16];
  f[13] = f[18];
  f[14] = f[18];
  f[15] = f[16];
  f[17] = f[18];
  f[19] = f[23];
  f[20] = f[23];
  f[21] = f[23];
  f[22] = f[23];
  f[24] = f[23];
  f[25] = f[23];
  f[26] = f[23];
}

// ---- outer normal (-1,+1,-1): 19 unknown populations ----
template <typename T>
PSL_HDI void mbbc_n6(T (&f)[27], const T rho, const T ux, const T uy, const T uz) {
  const T smf0 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(f[0], f[2]), f[3]), f[6]), f[10]), f[13]), f[15]), f[19]);
  const T smf1 = rn_sub(rn_sub(rn_sub((-f[2]), f[10]), f[15]), f[19]);
  const T smf2 = rn_add(rn_add(rn_add(f[6], f[13]), f[15]), f[19]);
  const T smf3 = rn_sub(rn_sub(rn_sub((-f[3]), f[10]), f[13]), f[19]);
  const T smf4 = rn_add(rn_add(rn_add(f[2], f[10]), f[15]), f[19]);
  const T smf5 = rn_add(rn_add(rn_add(f[6], f[13]), f[15]), f[19]);
  const T smf6 = rn_add(rn_add(rn_add(f[3], f[10]), f[13]), f[19]);
  const T smf7 = rn_sub((-f[13]), f[19]);
  const T smf8 = rn_add(f[10], f[19]);
  const T smf9 = rn_sub((-f[15]), f[19]);
  const T smf10 = rn_add(f[15], f[19]);
  const T smf11 = rn_sub((-f[10]), f[19]);
  const T smf12 = rn_sub((-f[15]), f[19]);
  const T smf13 = rn_sub((-f[13]), f[19]);
  const T smf14 = rn_sub((-f[10]), f[19]);
  const T smf15 = rn_add(f[13], f[19]);
  const T smf16 = rn_add(f[13], f[19]);
  const T smf17 = rn_add(f[10], f[19]);
  const T smf18 = rn_add(f[15], f[19]);
  const T m0 = rho;
  const T m1 = rn_mul(rho, ux);
  const T m2 = rn_mul(rho, uy);
  const T m3 = rn_mul(rho, uz);
  const T m4 = rn_add(rn_mul((T(1) / T(3)), rho), rn_mul(rn_mul(rho, ux), ux));
  const T m5 = rn_add(rn_mul((T(1) / T(3)), rho), rn_mul(rn_mul(rho, uy), uy));
  const T m6 = rn_add(rn_mul((T(1) / T(3)), rho), rn_mul(rn_mul(rho, uz), uz));
  const T m7 = rn_mul(rn_mul(rho, uy), uz);
  const T m8 = rn_mul(rn_mul(rho, ux), uz);
  const T m9 = rn_mul(rn_mul(rho, ux), uy);
  const T m10 = rn_add(rn_mul(rn_mul((T(1) / T(3)), rho), uy), rn_mul(rn_mul(rn_mul(rho, ux), ux), uy));
  const T m11 = rn_add(rn_mul(rn_mul((T(1) / T(3)), rho), uz), rn_mul(rn_mul(rn_mul(rho, ux), ux), uz));
  const T m12 = rn_add(rn_mul(rn_mul((T(1) / T(3)), rho), ux), rn_mul(rn_mul(rn_mul(rho, ux), uy), uy));
  const T m13 = rn_add(rn_mul(rn_mul((T(1) / T(3)), rho), uz), rn_mul(rn_mul(rn_mul(rho, uy), uy), uz));
  const T m14 = rn_add(rn_mul(rn_mul((T(1) / T(3)), rho), ux), rn_mul(rn_mul(rn_mul(rho, ux), uz), uz));
  const T m15 = rn_add(rn_mul(rn_mul((T(1) / T(3)), rho), uy), rn_mul(rn_mul(rn_mul(rho, uy), uz), uz));
  const T m16 = rn_add(rn_add(rn_add(rn_mul((T(1) / T(9)), rho), rn_mul(rn_mul(rn_mul((T(1) / T(3)), rho), uy), uy)), rn_mul(rn_mul(rn_mul((T(1) / T(3)), rho), uz), uz)), rn_mul(rn_mul(rn_mul(rn_mul(rho, uy), uy), uz), uz));
  const T m17 = rn_add(rn_add(rn_add(rn_mul((T(1) / T(9)), rho), rn_mul(rn_mul(rn_mul((T(1) / T(3)), rho), ux), ux)), rn_mul(rn_mul(rn_mul((T(1) / T(3)), rho), uz), uz)), rn_mul(rn_mul(rn_mul(rn_mul(rho, ux), ux), uz), uz));
  const T m18 = rn_add(rn_add(rn_add(rn_mul((T(1) / T(9)), rho), rn_mul(rn_mul(rn_mul((T(1) / T(3)), rho), ux), ux)), rn_mul(rn_mul(rn_mul((T(1) / T(3)), rho), uy), uy)), rn_mul(rn_mul(rn_mul(rn_mul(rho, ux), ux), uy), uy));
  const T s0 = rn_sub(m0, smf0);
  const T s1 = rn_sub(m1, smf1);
  const T s2 = rn_sub(m2, smf2);
  const T s3 = rn_sub(m3, smf3);
  const T s4 = rn_sub(m4, smf4);
  const T s5 = rn_sub(m5, smf5);
  const T s6 = rn_sub(m6, smf6);
  const T s7 = rn_sub(m7, smf7);
  const T s8 = rn_sub(m8, smf8);
  const T s9 = rn_sub(m9, smf9);
  const T s10 = rn_sub(m10, smf10);
  const T s11 = rn_sub(m11, smf11);
  const T s12 = rn_sub(m12, smf12);
  const T s13 = rn_sub(m13, smf13);
  const T s14 = rn_sub(m14, smf14);
  const T s15 = rn_sub(m15, smf15);
  const T s16 = rn_sub(m16, smf16);
  const T s17 = rn_sub(m17, smf17);
  const T s18 = rn_sub(m18, smf18);
  f[1] = rn_add(rn_sub(rn_sub(s0, s5), s6), s16);
  f[4] = rn_add(rn_sub(rn_sub(s0, s4), s5), s18);
  f[5] = rn_add(rn_sub(rn_sub(s0, s4), s6), s17);
  f[7] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(2)), s3), rn_mul((T(1) / T(2)), s6)), rn_mul((T(1) / T(2)), s13)), rn_mul((T(-1) / T(2)), s16));
  f[8] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(2)), s1), rn_mul((T(1) / T(2)), s4)), rn_mul((T(1) / T(2)), s12)), rn_mul((T(-1) / T(2)), s18));
  f[9] = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add((-s0), rn_mul((T(1) / T(2)), s1)), rn_mul((T(1) / T(2)), s3)), rn_mul((T(1) / T(2)), s4)), s5), rn_mul((T(1) / T(2)), s6)), rn_mul((T(-1) / T(2)), s12)), rn_mul((T(-1) / T(2)), s13)), rn_mul((T(-1) / T(2)), s16)), rn_mul((T(-1) / T(2)), s18));
  f[11] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(2)), s1), rn_mul((T(1) / T(2)), s4)), rn_mul((T(1) / T(2)), s14)), rn_mul((T(-1) / T(2)), s17));
  f[12] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), s2), rn_mul((T(1) / T(2)), s5)), rn_mul((T(-1) / T(2)), s15)), rn_mul((T(-1) / T(2)), s16));
  f[14] = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add((-s0), rn_mul((T(-1) / T(2)), s2)), rn_mul((T(1) / T(2)), s3)), s4), rn_mul((T(1) / T(2)), s5)), rn_mul((T(1) / T(2)), s6)), rn_mul((T(1) / T(2)), s10)), rn_mul((T(-1) / T(2)), s11)), rn_mul((T(-1) / T(2)), s17)), rn_mul((T(-1) / T(2)), s18));
  f[16] = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add((-s0), rn_mul((T(1) / T(2)), s1)), rn_mul((T(-1) / T(2)), s2)), rn_mul((T(1) / T(2)), s4)), rn_mul((T(1) / T(2)), s5)), s6), rn_mul((T(-1) / T(2)), s14)), rn_mul((T(1) / T(2)), s15)), rn_mul((T(-1) / T(2)), s16)), rn_mul((T(-1) / T(2)), s17));
  f[17] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), s2), rn_mul((T(1) / T(2)), s5)), rn_mul((T(-1) / T(2)), s10)), rn_mul((T(-1) / T(2)), s18));
  f[18] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(2)), s3), rn_mul((T(1) / T(2)), s6)), rn_mul((T(1) / T(2)), s11)), rn_mul((T(-1) / T(2)), s17));
  f[20] = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(s0, rn_mul((T(-1) / T(2)), s1)), rn_mul((T(1) / T(2)), s2)), rn_mul((T(-1) / T(2)), s3)), rn_mul((T(-1) / T(2)), s4)), rn_mul((T(-1) / T(2)), s5)), rn_mul((T(-1) / T(2)), s6)), rn_mul((T(-1) / T(4)), s7)), rn_mul((T(1) / T(4)), s8)), rn_mul((T(-1) / T(4)), s9)), rn_mul((T(-1) / T(4)), s10)), rn_mul((T(1) / T(4)), s11)), rn_mul((T(1) / T(4)), s12)), rn_mul((T(1) / T(4)), s13)), rn_mul((T(1) / T(4)), s14)), rn_mul((T(-1) / T(4)), s15)), rn_mul((T(1) / T(4)), s16)), rn_mul((T(1) / T(4)), s17)), rn_mul((T(1) / T(4)), s18));
  f[21] = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), s1), rn_mul((T(-1) / T(2)), s4)), rn_mul((T(-1) / T(4)), s8)), rn_mul((T(1) / T(4)), s9)), rn_mul((T(-1) / T(4)), s10)), rn_mul((T(1) / T(4)), s11)), rn_mul((T(-1) / T(4)), s12)), rn_mul((T(-1) / T(4)), s14)), rn_mul((T(1) / T(4)), s17)), rn_mul((T(1) / T(4)), s18));
  f[22] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(4)), s7), rn_mul((T(-1) / T(4)), s13)), rn_mul((T(1) / T(4)), s15)), rn_mul((T(1) / T(4)), s16));
  f[23] = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), s3), rn_mul((T(-1) / T(2)), s6)), rn_mul((T(1) / T(4)), s7)), rn_mul((T(-1) / T(4)), s8)), rn_mul((T(-1) / T(4)), s11)), rn_mul((T(-1) / T(4)), s13)), rn_mul((T(1) / T(4)), s14)), rn_mul((T(-1) / T(4)), s15)), rn_mul((T(1) / T(4)), s16)), rn_mul((T(1) / T(4)), s17));
  f[24] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(4)), s9), rn_mul((T(1) / T(4)), s10)), rn_mul((T(-1) / T(4)), s12)), rn_mul((T(1) / T(4)), s18));
  f[25] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(4)), s8), rn_mul((T(-1) / T(4)), s11)), rn_mul((T(-1) / T(4)), s14)), rn_mul((T(1) / T(4)), s17));
  f[26] = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_mul((T(-1) / T(2)), s2), rn_mul((T(-1) / T(2)), s5)), rn_mul((T(1) / T(4)), s7)), rn_mul((T(1) / T(4)), s9)), rn_mul((T(1) / T(4)), s10)), rn_mul((T(1) / T(4)), s12)), rn_mul((T(1) / T(4)), s13)), rn_mul((T(1) / T(4)), s15)), rn_mul((T(1) / T(4)), s16)), rn_mul((T(1) / T(4)), s18));
}
template <typename T>
PSL_HDI void restore_rho_u_n6(const T (&f)[27], T& rho, T& ux, T& uy, T& uz) {
  const T q0 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_mul((T(5) / T(2)), f[0]), rn_mul(T(2), f[2])), rn_mul(T(2), f[3])), rn_mul(T(2), f[6])), rn_mul(T(-2), f[10])), rn_mul(T(-2), f[13])), rn_mul(T(-2), f[15])), rn_mul(T(-16), f[19]));
  const T q1 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), f[0]), rn_mul(T(-2), f[2])), f[3]), f[6]), rn_mul(T(-4), f[10])), rn_mul(T(2), f[13])), rn_mul(T(-4), f[15])), rn_mul(T(-8), f[19]));
  const T q2 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_sub(rn_sub(rn_mul((T(-1) / T(2)), f[0]), f[2]), f[3]), rn_mul(T(2), f[6])), rn_mul(T(-2), f[10])), rn_mul(T(4), f[13])), rn_mul(T(4), f[15])), rn_mul(T(8), f[19]));
  const T q3 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), f[0]), f[2]), rn_mul(T(-2), f[3])), f[6]), rn_mul(T(-4), f[10])), rn_mul(T(-4), f[13])), rn_mul(T(2), f[15])), rn_mul(T(-8), f[19]));
  rho = q0;
  ux = rn_div(q1, rho);
  uy = rn_div(q2, rho);
  uz = rn_div(q3, rho);
}
template <typename T>
PSL_HDI void restore_u_n6(const T (&f)[27], const T rho, T& ux, T& uy, T& uz) {
  const T scmf0 = rn_div(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(f[0], rn_mul(T(2), f[2])), rn_mul(T(2), f[3])), rn_mul(T(2), f[6])), rn_mul(T(4), f[10])), rn_mul(T(4), f[13])), rn_mul(T(4), f[15])), rn_mul(T(8), f[19])), rho);
  const T scmf1 = rn_div(rn_add(rn_add(rn_add(f[0], rn_mul(T(2), f[3])), rn_mul(T(2), f[6])), rn_mul(T(4), f[13])), rho);
  const T scmf2 = rn_div(rn_add(rn_add(rn_add((-f[0]), rn_mul(T(-2), f[2])), rn_mul(T(-2), f[3])), rn_mul(T(-4), f[10])), rho);
  const T s0 = rn_sub(scmf0, T(1));
  const T s1 = rn_sub(scmf1, (T(2) / T(3)));
  const T s2 = rn_sub(scmf2, (T(-2) / T(3)));
  ux = rn_add((-s0), rn_mul((T(3) / T(2)), s1));
  uy = rn_add(s0, rn_mul((T(3) / T(2)), s2));
  uz = rn_add(rn_add(s0, rn_mul((T(-3) / T(2)), s1)), rn_mul((T(3) / T(2)), s2));
}
template <typename T>
PSL_HDI void restore_rho_n6(const T (&f)[27], T& rho, const T ux, const T uy, const T uz) {
  const T scqu = rn_add(rn_add(rn_mul(T(-1), ux), rn_mul(T(1), uy)), rn_mul(T(-1), uz));
  const T s = rn_add(T(1), scqu);
  const T scmf = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(f[0], rn_mul(T(2), f[2])), rn_mul(T(2), f[3])), rn_mul(T(2), f[6])), rn_mul(T(4), f[10])), rn_mul(T(4), f[13])), rn_mul(T(4), f[15])), rn_mul(T(8), f[19]));
  rho = rn_div(scmf, s);
}
template <typename T>
PSL_HDI void mirror_n6(T (&f)[27]) {
  f[1] = f[2];
  f[4] = f[3];
  f[5] = f[6];
  f[7] = f[10];
  f[8] = f[10];
  f[9] = f[10];
  f[11] = f[15];
  f[12] = f[15];
  f[14] = f[13];
  f[16] = f[15];
  f[17] = f[13];
  f[18] = f[13];
  f[20] = f[19];
  f[21] = f[19];
  f[22] = f[19];
  f[23] = f[19];
  f[24] = f[19];
  f[25] = f[19];
  f[26] = f[19];
}

// ---- outer normal (-1,-1,+1): 19 unknown populations ----
template <typename T>
PSL_HDI void mbbc_n2(T (&f)[27], const T rho, const T ux, const T uy, const T uz) {
  const T smf0 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(f[0], f[2]), f[4]), f[5]), f[8]), f[11]), f[14]), f[21]);
  const T smf1 = rn_sub(rn_sub(rn_sub((-f[2]), f[8]), f[11]), f[21]);
  const T smf2 = rn_sub(rn_sub(rn_sub((-f[5]), f[11]), f[14]), f[21]);
  const T smf3 = rn_add(rn_add(rn_add(f[4], f[8]), f[14]), f[21]);
  const T smf4 = rn_add(rn_add(rn_add(f[2], f[8]), f[11]), f[21]);
  const T smf5 = rn_add(rn_add(rn_add(f[5], f[11]), f[14]), f[21]);
  const T smf6 = rn_add(rn_add(rn_add(f[4], f[8]), f[14]), f[21]);
  const T smf7 = rn_sub((-f[14]), f[21]);
  const T smf8 = rn_sub((-f[8]), f[21]);
  const T smf9 = rn_add(f[11], f[21]);
  const T smf10 = rn_sub((-f[11]), f[21]);
  const T smf11 = rn_add(f[8], f[21]);
  const T smf12 = rn_sub((-f[11]), f[21]);
  const T smf13 = rn_add(f[14], f[21]);
  const T smf14 = rn_sub((-f[8]), f[21]);
  const T smf15 = rn_sub((-f[14]), f[21]);
  const T smf16 = rn_add(f[14], f[21]);
  const T smf17 = rn_add(f[8], f[21]);
  const T smf18 = rn_add(f[11], f[21]);
  const T m0 = rho;
  const T m1 = rn_mul(rho, ux);
  const T m2 = rn_mul(rho, uy);
  const T m3 = rn_mul(rho, uz);
  const T m4 = rn_add(rn_mul((T(1) / T(3)), rho), rn_mul(rn_mul(rho, ux), ux));
  const T m5 = rn_add(rn_mul((T(1) / T(3)), rho), rn_mul(rn_mul(rho, uy), uy));
  const T m6 = rn_add(rn_mul((T(1) / T(3)), rho), rn_mul(rn_mul(rho, uz), uz));
  const T m7 = rn_mul(rn_mul(rho, uy), uz);
  const T m8 = rn_mul(rn_mul(rho, ux), uz);
  const T m9 = rn_mul(rn_mul(rho, ux), uy);
  const T m10 = rn_add(rn_mul(rn_mul((T(1) / T(3)), rho), uy), rn_mul(rn_mul(rn_mul(rho, ux), ux), uy));
  const T m11 = rn_add(rn_mul(rn_mul((T(1) / T(3)), rho), uz), rn_mul(rn_mul(rn_mul(rho, ux), ux), uz));
  const T m12 = rn_add(rn_mul(rn_mul((T(1) / T(3)), rho), ux), rn_mul(rn_mul(rn_mul(rho, ux), uy), uy));
  const T m13 = rn_add(rn_mul(rn_mul((T(1) / T(3)), rho), uz), rn_mul(rn_mul(rn_mul(rho, uy), uy), uz));
  const T m14 = rn_add(rn_mul(rn_mul((T(1) / T(3)), rho), ux), rn_mul(rn_mul(rn_mul(rho, ux), uz), uz));
  const T m15 = rn_add(rn_mul(rn_mul((T(1) / T(3)), rho), uy), rn_mul(rn_mul(rn_mul(rho, uy), uz), uz));
  const T m16 = rn_add(rn_add(rn_add(rn_mul((T(1) / T(9)), rho), rn_mul(rn_mul(rn_mul((T(1) / T(3)), rho), uy), uy)), rn_mul(rn_mul(rn_mul((T(1) / T(3)), rho), uz), uz)), rn_mul(rn_mul(rn_mul(rn_mul(rho, uy), uy), uz), uz));
  const T m17 = rn_add(rn_add(rn_add(rn_mul((T(1) / T(9)), rho), rn_mul(rn_mul(rn_mul((T(1) / T(3)), rho), ux), ux)), rn_mul(rn_mul(rn_mul((T(1) / T(3)), rho), uz), uz)), rn_mul(rn_mul(rn_mul(rn_mul(rho, ux), ux), uz), uz));
  const T m18 = rn_add(rn_add(rn_add(rn_mul((T(1) / T(9)), rho), rn_mul(rn_mul(rn_mul((T(1) / T(3)), rho), ux), ux)), rn_mul(rn_mul(rn_mul((T(1) / T(3)), rho), uy), uy)), rn_mul(rn_mul(rn_mul(rn_mul(rho, ux), ux), uy), uy));
  const T s0 = rn_sub(m0, smf0);
  const T s1 = rn_sub(m1, smf1);
  const T s2 = rn_sub(m2, smf2);
  const T s3 = rn_sub(m3, smf3);
  const T s4 = rn_sub(m4, smf4);
  const T s5 = rn_sub(m5, smf5);
  const T s6 = rn_sub(m6, smf6);
  const T s7 = rn_sub(m7, smf7);
  const T s8 = rn_sub(m8, smf8);
  const T s9 = rn_sub(m9, smf9);
  const T s10 = rn_sub(m10, smf10);
  const T s11 = rn_sub(m11, smf11);
  const T s12 = rn_sub(m12, smf12);
  const T s13 = rn_sub(m13, smf13);
  const T s14 = rn_sub(m14, smf14);
  const T s15 = rn_sub(m15, smf15);
  const T s16 = rn_sub(m16, smf16);
  const T s17 = rn_sub(m17, smf17);
  const T s18 = rn_sub(m18, smf18);
  f[1] = rn_add(rn_sub(rn_sub(s0, s5), s6), s16);
  f[3] = rn_add(rn_sub(rn_sub(s0, s4), s5), s18);
  f[6] = rn_add(rn_sub(rn_sub(s0, s4), s6), s17);
  f[7] = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add((-s0), rn_mul((T(1) / T(2)), s1)), rn_mul((T(-1) / T(2)), s3)), rn_mul((T(1) / T(2)), s4)), s5), rn_mul((T(1) / T(2)), s6)), rn_mul((T(-1) / T(2)), s12)), rn_mul((T(1) / T(2)), s13)), rn_mul((T(-1) / T(2)), s16)), rn_mul((T(-1) / T(2)), s18));
  f[9] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), s3), rn_mul((T(1) / T(2)), s6)), rn_mul((T(-1) / T(2)), s13)), rn_mul((T(-1) / T(2)), s16));
  f[10] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(2)), s1), rn_mul((T(1) / T(2)), s4)), rn_mul((T(1) / T(2)), s12)), rn_mul((T(-1) / T(2)), s18));
  f[12] = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add((-s0), rn_mul((T(1) / T(2)), s1)), rn_mul((T(1) / T(2)), s2)), rn_mul((T(1) / T(2)), s4)), rn_mul((T(1) / T(2)), s5)), s6), rn_mul((T(-1) / T(2)), s14)), rn_mul((T(-1) / T(2)), s15)), rn_mul((T(-1) / T(2)), s16)), rn_mul((T(-1) / T(2)), s17));
  f[13] = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add((-s0), rn_mul((T(1) / T(2)), s2)), rn_mul((T(-1) / T(2)), s3)), s4), rn_mul((T(1) / T(2)), s5)), rn_mul((T(1) / T(2)), s6)), rn_mul((T(-1) / T(2)), s10)), rn_mul((T(1) / T(2)), s11)), rn_mul((T(-1) / T(2)), s17)), rn_mul((T(-1) / T(2)), s18));
  f[15] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(2)), s1), rn_mul((T(1) / T(2)), s4)), rn_mul((T(1) / T(2)), s14)), rn_mul((T(-1) / T(2)), s17));
  f[16] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(2)), s2), rn_mul((T(1) / T(2)), s5)), rn_mul((T(1) / T(2)), s15)), rn_mul((T(-1) / T(2)), s16));
  f[17] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), s3), rn_mul((T(1) / T(2)), s6)), rn_mul((T(-1) / T(2)), s11)), rn_mul((T(-1) / T(2)), s17));
  f[18] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(2)), s2), rn_mul((T(1) / T(2)), s5)), rn_mul((T(1) / T(2)), s10)), rn_mul((T(-1) / T(2)), s18));
  f[19] = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), s1), rn_mul((T(-1) / T(2)), s4)), rn_mul((T(1) / T(4)), s8)), rn_mul((T(-1) / T(4)), s9)), rn_mul((T(1) / T(4)), s10)), rn_mul((T(-1) / T(4)), s11)), rn_mul((T(-1) / T(4)), s12)), rn_mul((T(-1) / T(4)), s14)), rn_mul((T(1) / T(4)), s17)), rn_mul((T(1) / T(4)), s18));
  f[20] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(4)), s7), rn_mul((T(1) / T(4)), s13)), rn_mul((T(-1) / T(4)), s15)), rn_mul((T(1) / T(4)), s16));
  f[22] = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(s0, rn_mul((T(-1) / T(2)), s1)), rn_mul((T(-1) / T(2)), s2)), rn_mul((T(1) / T(2)), s3)), rn_mul((T(-1) / T(2)), s4)), rn_mul((T(-1) / T(2)), s5)), rn_mul((T(-1) / T(2)), s6)), rn_mul((T(-1) / T(4)), s7)), rn_mul((T(-1) / T(4)), s8)), rn_mul((T(1) / T(4)), s9)), rn_mul((T(1) / T(4)), s10)), rn_mul((T(-1) / T(4)), s11)), rn_mul((T(1) / T(4)), s12)), rn_mul((T(-1) / T(4)), s13)), rn_mul((T(1) / T(4)), s14)), rn_mul((T(1) / T(4)), s15)), rn_mul((T(1) / T(4)), s16)), rn_mul((T(1) / T(4)), s17)), rn_mul((T(1) / T(4)), s18));
  f[23] = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), s2), rn_mul((T(-1) / T(2)), s5)), rn_mul((T(1) / T(4)), s7)), rn_mul((T(-1) / T(4)), s9)), rn_mul((T(-1) / T(4)), s10)), rn_mul((T(1) / T(4)), s12)), rn_mul((T(-1) / T(4)), s13)), rn_mul((T(-1) / T(4)), s15)), rn_mul((T(1) / T(4)), s16)), rn_mul((T(1) / T(4)), s18));
  f[24] = rn_add(rn_add(rn_add(rn_mul((T(-1) / T(4)), s8), rn_mul((T(1) / T(4)), s11)), rn_mul((T(-1) / T(4)), s14)), rn_mul((T(1) / T(4)), s17));
  f[25] = rn_add(rn_add(rn_add(rn_mul((T(1) / T(4)), s9), rn_mul((T(-1) / T(4)), s10)), rn_mul((T(-1) / T(4)), s12)), rn_mul((T(1) / T(4)), s18));
  f[26] = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_mul((T(-1) / T(2)), s3), rn_mul((T(-1) / T(2)), s6)), rn_mul((T(1) / T(4)), s7)), rn_mul((T(1) / T(4)), s8)), rn_mul((T(1) / T(4)), s11)), rn_mul((T(1) / T(4)), s13)), rn_mul((T(1) / T(4)), s14)), rn_mul((T(1) / T(4)), s15)), rn_mul((T(1) / T(4)), s16)), rn_mul((T(1) / T(4)), s17));
}
template <typename T>
PSL_HDI void restore_rho_u_n2(const T (&f)[27], T& rho, T& ux, T& uy, T& uz) {
  const T q0 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_mul((T(5) / T(2)), f[0]), rn_mul(T(2), f[2])), rn_mul(T(2), f[4])), rn_mul(T(2), f[5])), rn_mul(T(-2), f[8])), rn_mul(T(-2), f[11])), rn_mul(T(-2), f[14])), rn_mul(T(-16), f[21]));
  const T q1 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), f[0]), rn_mul(T(-2), f[2])), f[4]), f[5]), rn_mul(T(-4), f[8])), rn_mul(T(-4), f[11])), rn_mul(T(2), f[14])), rn_mul(T(-8), f[21]));
  const T q2 = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_mul((T(1) / T(2)), f[0]), f[2]), f[4]), rn_mul(T(-2), f[5])), rn_mul(T(2), f[8])), rn_mul(T(-4), f[11])), rn_mul(T(-4), f[14])), rn_mul(T(-8), f[21]));
  const T q3 = rn_add(rn_add(rn_add(rn_add(rn_sub(rn_add(rn_sub(rn_mul((T(-1) / T(2)), f[0]), f[2]), rn_mul(T(2), f[4])), f[5]), rn_mul(T(4), f[8])), rn_mul(T(-2), f[11])), rn_mul(T(4), f[14])), rn_mul(T(8), f[21]));
  rho = q0;
  ux = rn_div(q1, rho);
  uy = rn_div(q2, rho);
  uz = rn_div(q3, rho);
}
template <typename T>
PSL_HDI void restore_u_n2(const T (&f)[27], const T rho, T& ux, T& uy, T& uz) {
  const T scmf0 = rn_div(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(f[0], rn_mul(T(2), f[2])), rn_mul(T(2), f[4])), rn_mul(T(2), f[5])), rn_mul(T(4), f[8])), rn_mul(T(4), f[11])), rn_mul(T(4), f[14])), rn_mul(T(8), f[21])), rho);
  const T scmf1 = rn_div(rn_add(rn_add(rn_add(f[0], rn_mul(T(2), f[4])), rn_mul(T(2), f[5])), rn_mul(T(4), f[14])), rho);
  const T scmf2 = rn_div(rn_add(rn_add(rn_add(f[0], rn_mul(T(2), f[2])), rn_mul(T(2), f[4])), rn_mul(T(4), f[8])), rho);
  const T s0 = rn_sub(scmf0, T(1));
  const T s1 = rn_sub(scmf1, (T(2) / T(3)));
  const T s2 = rn_sub(scmf2, (T(2) / T(3)));
  ux = rn_add((-s0), rn_mul((T(3) / T(2)), s1));
  uy = rn_add((-s0), rn_mul((T(3) / T(2)), s2));
  uz = rn_add(rn_add((-s0), rn_mul((T(3) / T(2)), s1)), rn_mul((T(3) / T(2)), s2));
}
template <typename T>
PSL_HDI void restore_rho_n2(const T (&f)[27], T& rho, const T ux, const T uy, const T uz) {
  const T scqu = rn_add(rn_add(rn_mul(T(-1), ux), rn_mul(T(-1), uy)), rn_mul(T(1), uz));
  const T s = rn_add(T(1), scqu);
  const T scmf = rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(rn_add(f[0], rn_mul(T(2), f[2])), rn_mul(T(2), f[4])), rn_mul(T(2), f[5])), rn_mul(T(4), f[8])), rn_mul(T(4), f[11])), rn_mul(T(4), f[14])), rn_mul(T(8), f[21]));
  rho = rn_div(scmf, s);
}
template <typename T>
PSL_HDI void mirror_n2(T (&f)[27]) {
  f[1] = f[2];
  f[3] = f[4];
  f[6] = f[5];
  f[7] = f[8];
  f[9] = f[8];
  f[10] = f[8];
  f[12] = f[11];
  f[13] = f[14];
  f[15] = f[11];
  f[16] = f[11];
  f[17] = f[14];
  f[18] = f[14];
  f[19] = f[21];
  f[20] = f[21];
  f[22] = f[21];
  f[23] = f[21];
  f[24] = f[21];
  f[25] = f[21];
  f[26] = f[21];
}

template <typename T>
PSL_HDI void mbbc(const int normal, T (&f)[27], const T rho, const T ux, const T uy, const T uz) {
  switch (normal) {
    case 22: mbbc_n22(f, rho, ux, uy, uz); break;
    case 16: mbbc_n16(f, rho, ux, uy, uz); break;
    case 14: mbbc_n14(f, rho, ux, uy, uz); break;
    case 4: mbbc_n4(f, rho, ux, uy, uz); break;
    case 10: mbbc_n10(f, rho, ux, uy, uz); break;
    case 12: mbbc_n12(f, rho, ux, uy, uz); break;
    case 17: mbbc_n17(f, rho, ux, uy, uz); break;
    case 23: mbbc_n23(f, rho, ux, uy, uz); break;
    case 25: mbbc_n25(f, rho, ux, uy, uz); break;
    case 9: mbbc_n9(f, rho, ux, uy, uz); break;
    case 3: mbbc_n3(f, rho, ux, uy, uz); break;
    case 1: mbbc_n1(f, rho, ux, uy, uz); break;
    case 15: mbbc_n15(f, rho, ux, uy, uz); break;
    case 21: mbbc_n21(f, rho, ux, uy, uz); break;
    case 19: mbbc_n19(f, rho, ux, uy, uz); break;
    case 11: mbbc_n11(f, rho, ux, uy, uz); break;
    case 5: mbbc_n5(f, rho, ux, uy, uz); break;
    case 7: mbbc_n7(f, rho, ux, uy, uz); break;
    case 26: mbbc_n26(f, rho, ux, uy, uz); break;
    case 0: mbbc_n0(f, rho, ux, uy, uz); break;
    case 8: mbbc_n8(f, rho, ux, uy, uz); break;
    case 20: mbbc_n20(f, rho, ux, uy, uz); break;
    case 24: mbbc_n24(f, rho, ux, uy, uz); break;
    case 18: mbbc_n18(f, rho, ux, uy, uz); break;
    case 6: mbbc_n6(f, rho, ux, uy, uz); break;
    case 2: mbbc_n2(f, rho, ux, uy, uz); break;
    default: break;
  }
}
template <typename T>
PSL_HDI void restore_rho_u(const int normal, const T (&f)[27], T& rho, T& ux, T& uy, T& uz) {
  switch (normal) {
    case 22: restore_rho_u_n22(f, rho, ux, uy, uz); break;
    case 16: restore_rho_u_n16(f, rho, ux, uy, uz); break;
    case 14: restore_rho_u_n14(f, rho, ux, uy, uz); break;
    case 4: restore_rho_u_n4(f, rho, ux, uy, uz); break;
    case 10: restore_rho_u_n10(f, rho, ux, uy, uz); break;
    case 12: restore_rho_u_n12(f, rho, ux, uy, uz); break;
    case 17: restore_rho_u_n17(f, rho, ux, uy, uz); break;
    case 23: restore_rho_u_n23(f, rho, ux, uy, uz); break;
    case 25: restore_rho_u_n25(f, rho, ux, uy, uz); break;
    case 9: restore_rho_u_n9(f, rho, ux, uy, uz); break;
    case 3: restore_rho_u_n3(f, rho, ux, uy, uz); break;
    case 1: restore_rho_u_n1(f, rho, ux, uy, uz); break;
    case 15: restore_rho_u_n15(f, rho, ux, uy, uz); break;
    case 21: restore_rho_u_n21(f, rho, ux, uy, uz); break;
    case 19: restore_rho_u_n19(f, rho, ux, uy, uz); break;
    case 11: restore_rho_u_n11(f, rho, ux, uy, uz); break;
    case 5: restore_rho_u_n5(f, rho, ux, uy, uz); break;
    case 7: restore_rho_u_n7(f, rho, ux, uy, uz); break;
    case 26: restore_rho_u_n26(f, rho, ux, uy, uz); break;
    case 0: restore_rho_u_n0(f, rho, ux, uy, uz); break;
    case 8: restore_rho_u_n8(f, rho, ux, uy, uz); break;
    case 20: restore_rho_u_n20(f, rho, ux, uy, uz); break;
    case 24: restore_rho_u_n24(f, rho, ux, uy, uz); break;
    case 18: restore_rho_u_n18(f, rho, ux, uy, uz); break;
    case 6: restore_rho_u_n6(f, rho, ux, uy, uz); break;
    case 2: restore_rho_u_n2(f, rho, ux, uy, uz); break;
    default: break;
  }
}
template <typename T>
PSL_HDI void restore_u(const int normal, const T (&f)[27], const T rho, T& ux, T& uy, T& uz) {
  switch (normal) {
    case 22: restore_u_n22(f, rho, ux, uy, uz); break;
    case 16: restore_u_n16(f, rho, ux, uy, uz); break;
    case 14: restore_u_n14(f, rho, ux, uy, uz); break;
    case 4: restore_u_n4(f, rho, ux, uy, uz); break;
    case 10: restore_u_n10(f, rho, ux, uy, uz); break;
    case 12: restore_u_n12(f, rho, ux, uy, uz); break;
    case 17: restore_u_n17(f, rho, ux, uy, uz); break;
    case 23: restore_u_n23(f, rho, ux, uy, uz); break;
    case 25: restore_u_n25(f, rho, ux, uy, uz); break;
    case 9: restore_u_n9(f, rho, ux, uy, uz); break;
    case 3: restore_u_n3(f, rho, ux, uy, uz); break;
    case 1: restore_u_n1(f, rho, ux, uy, uz); break;
    case 15: restore_u_n15(f, rho, ux, uy, uz); break;
    case 21: restore_u_n21(f, rho, ux, uy, uz); break;
    case 19: restore_u_n19(f, rho, ux, uy, uz); break;
    case 11: restore_u_n11(f, rho, ux, uy, uz); break;
    case 5: restore_u_n5(f, rho, ux, uy, uz); break;
    case 7: restore_u_n7(f, rho, ux, uy, uz); break;
    case 26: restore_u_n26(f, rho, ux, uy, uz); break;
    case 0: restore_u_n0(f, rho, ux, uy, uz); break;
    case 8: restore_u_n8(f, rho, ux, uy, uz); break;
    case 20: restore_u_n20(f, rho, ux, uy, uz); break;
    case 24: restore_u_n24(f, rho, ux, uy, uz); break;
    case 18: restore_u_n18(f, rho, ux, uy, uz); break;
    case 6: restore_u_n6(f, rho, ux, uy, uz); break;
    case 2: restore_u_n2(f, rho, ux, uy, uz); break;
    default: break;
  }
}
template <typename T>
PSL_HDI void restore_rho(const int normal, const T (&f)[27], T& rho, const T ux, const T uy, const T uz) {
  switch (normal) {
    case 22: restore_rho_n22(f, rho, ux, uy, uz); break;
    case 16: restore_rho_n16(f, rho, ux, uy, uz); break;
    case 14: restore_rho_n14(f, rho, ux, uy, uz); break;
    case 4: restore_rho_n4(f, rho, ux, uy, uz); break;
    case 10: restore_rho_n10(f, rho, ux, uy, uz); break;
    case 12: restore_rho_n12(f, rho, ux, uy, uz); break;
    case 17: restore_rho_n17(f, rho, ux, uy, uz); break;
    case 23: restore_rho_n23(f, rho, ux, uy, uz); break;
    case 25: restore_rho_n25(f, rho, ux, uy, uz); break;
    case 9: restore_rho_n9(f, rho, ux, uy, uz); break;
    case 3: restore_rho_n3(f, rho, ux, uy, uz); break;
    case 1: restore_rho_n1(f, rho, ux, uy, uz); break;
    case 15: restore_rho_n15(f, rho, ux, uy, uz); break;
    case 21: restore_rho_n21(f, rho, ux, uy, uz); break;
    case 19: restore_rho_n19(f, rho, ux, uy, uz); break;
    case 11: restore_rho_n11(f, rho, ux, uy, uz); break;
    case 5: restore_rho_n5(f, rho, ux, uy, uz); break;
    case 7: restore_rho_n7(f, rho, ux, uy, uz); break;
    case 26: restore_rho_n26(f, rho, ux, uy, uz); break;
    case 0: restore_rho_n0(f, rho, ux, uy, uz); break;
    case 8: restore_rho_n8(f, rho, ux, uy, uz); break;
    case 20: restore_rho_n20(f, rho, ux, uy, uz); break;
    case 24: restore_rho_n24(f, rho, ux, uy, uz); break;
    case 18: restore_rho_n18(f, rho, ux, uy, uz); break;
    case 6: restore_rho_n6(f, rho, ux, uy, uz); break;
    case 2: restore_rho_n2(f, rho, ux, uy, uz); break;
    default: break;
  }
}
template <typename T>
PSL_HDI void mirror(const int normal, T (&f)[27]) {
  switch (normal) {
    case 22: mirror_n22(f); break;
    case 16: mirror_n16(f); break;
    case 14: mirror_n14(f); break;
    case 4: mirror_n4(f); break;
    case 10: mirror_n10(f); break;
    case 12: mirror_n12(f); break;
    case 17: mirror_n17(f); break;
    case 23: mirror_n23(f); break;
    case 25: mirror_n25(f); break;
    case 9: mirror_n9(f); break;
    case 3: mirror_n3(f); break;
    case 1: mirror_n1(f); break;
    case 15: mirror_n15(f); break;
    case 21: mirror_n21(f); break;
    case 19: mirror_n19(f); break;
    case 11: mirror_n11(f); break;
    case 5: mirror_n5(f); break;
    case 7: mirror_n7(f); break;
    case 26: mirror_n26(f); break;
    case 0: mirror_n0(f); break;
    case 8: mirror_n8(f); break;
    case 20: mirror_n20(f); break;
    case 24: mirror_n24(f); break;
    case 18: mirror_n18(f); break;
    case 6: mirror_n6(f); break;
    case 2: mirror_n2(f); break;
    default: break;
  }
}

}  // namespace bc
}  // namespace psl
