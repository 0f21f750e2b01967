// The cumulant collision of the 16-bit storage forms, evaluated on the stored deviations
// g_q = f_q - w_q directly (no f = g + w before the collision, no f - w after it).
//
// The "all-one" cumulant model (include/applyCollision.h:6-295, Geier et al. 2015) needs
// only the density, the momentum and the six second-order central moments of a cell:
// everything else it writes back is rebuilt from them (first-order central moments zero,
// relaxed second-order cumulants, third-order cumulants zero, fourth- and sixth-order
// central moments from products of the second-order ones).  So the forward side here is
// ten raw moments of g instead of the 27-entry central-moment transform:
//     rho = 1 + sum g            (sum w = 1)
//     j   = sum c g              (sum c w = 0)
//     S   = sum c c g            (sum c c w = I/3)
// and with D = C - (rho/3) I, the second-order central moments less their equilibrium
// part (C = M - rho u u exactly, M = S + I/3):
//     D_ab = S_ab - delta_ab (rho - 1)/3 - j_a u_b.
// D is computed from small quantities only, which is also what the 16-bit forms store.
//
// The backward transform (Geier 2015 eqs 88-96, per axis
//     f(-1) = m0 (u^2-u)/2 + m1 (u-1/2) + m2/2, f(0) = m0 (1-u^2) - 2u m1 - m2,
//     f(+1) = m0 (u^2+u)/2 + m1 (u+1/2) + m2/2)
// is written with h = m0 u^2/2 + u m1 + m2/2 and e = (u m0 + m1)/2:
//     f(-1) = h - e,  f(+1) = h + e,  f(0) = m0 - 2h,
// on inputs pre-scaled by 1/2 per non-zero order (m1' = m1/2, m2' = m2/2 at every pass,
// folded into the moments), so a full triple costs six operations; the lattice weights
// are subtracted inside the last pass, so the output is g' = f' - w.
//
// Same physics as collide<false> (psl_collision.cuh); results agree to FP32 rounding (the
// operation order differs, and the device takes the approximate reciprocal and square
// root).  Templated on the arithmetic type (float everywhere today; host-compilable,
// PSL_HDI, so the CPU tests can check it against the oracle's collision).
#pragma once
#include <math.h>
#if defined(__CUDACC__)
#include <cuda_fp16.h>
#endif

#include "psl_lattice.cuh"

namespace psl {

// The scalar forms of the operations the templates use.  On the device the reciprocal and
// the square root are the single-instruction approximations of PTX (rcp.approx, sqrt.approx:
// relative error of order 2^-23, far below the 16-bit forms' storage rounding of 2^-11 /
// 2^-8); host builds (the CPU checks of this header) divide and take sqrtf.
PSL_HDI float gfma(float a, float b, float c) { return fmaf(a, b, c); }
PSL_HDI float grecip(float a) {
#if defined(__CUDA_ARCH__)
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(a));
  return r;
#else
  return 1.f / a;
#endif
}
PSL_HDI float gsqrt(float a) {
#if defined(__CUDA_ARCH__)
  float r;
  asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(a));
  return r;
#else
  return sqrtf(a);
#endif
}
PSL_HDI bool all_zero(float a) { return a == 0.f; }
PSL_HDI float sel_zero(float c, float if_zero, float other) { return c == 0.f ? if_zero : other; }
PSL_HDI bool finite_density(float rho) { return rho > 0.f && rho < 1.0e30f; }

// Ten raw moments of g: rg = sum g, j = sum c g, S_ab = sum c_a c_b g.  z-lines first
// (3 ops per line), then y (8 per x-slot), then x (15): 66 additions.
template <typename T>
struct RawMomentsGT {
  T rg, jx, jy, jz, sxx, syy, szz, sxy, sxz, syz;
};

// The y and x stages from the z-line sums (z0: sum, z1: first moment, z2: second moment
// along z of each (x, y) line).
template <typename T>
PSL_HDI RawMomentsGT<T> raw_moments_from_z(const T (&z0)[3][3], const T (&z1)[3][3], const T (&z2)[3][3]) {
  T y00[3], y10[3], y20[3], y01[3], y11[3], y02[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    y20[i] = z0[i][2] + z0[i][0];
    y10[i] = z0[i][2] - z0[i][0];
    y00[i] = y20[i] + z0[i][1];
    y11[i] = z1[i][2] - z1[i][0];
    y01[i] = (z1[i][2] + z1[i][0]) + z1[i][1];
    y02[i] = (z2[i][2] + z2[i][0]) + z2[i][1];
  }
  RawMomentsGT<T> m;
  m.sxx = y00[2] + y00[0];
  m.jx = y00[2] - y00[0];
  m.rg = m.sxx + y00[1];
  m.jy = (y10[2] + y10[0]) + y10[1];
  m.sxy = y10[2] - y10[0];
  m.syy = (y20[2] + y20[0]) + y20[1];
  m.jz = (y01[2] + y01[0]) + y01[1];
  m.sxz = y01[2] - y01[0];
  m.syz = (y11[2] + y11[0]) + y11[1];
  m.szz = (y02[2] + y02[0]) + y02[1];
  return m;
}

template <typename T>
PSL_HDI RawMomentsGT<T> raw_moments_g(const T (&g)[27]) {
  T z0[3][3], z1[3][3], z2[3][3];
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      const T a = g[slot(i, j, 0)], b = g[slot(i, j, 1)], c = g[slot(i, j, 2)];
      z2[i][j] = c + a;
      z0[i][j] = z2[i][j] + b;
      z1[i][j] = c - a;
    }
  return raw_moments_from_z(z0, z1, z2);
}

#if defined(__CUDACC__)
// The same sums started from the stored 16-bit values.  add.f32.f16 / add.f32.bf16 (PTX,
// sm_100) convert their 16-bit operand and add in FP32 as one instruction; the conversion
// is exact, so every sum is the one raw_moments_g forms from the converted values, bit for
// bit (c - a is formed as -(a - c), the same rounding).
template <bool kBF16>
__device__ __forceinline__ float bits_to_float(uint16_t v) {
  if constexpr (kBF16) return __uint_as_float((uint32_t)v << 16);
  else return __half2float(__ushort_as_half(v));
}
template <bool kBF16>
__device__ __forceinline__ float add_bits(uint16_t a, float c) {
  float r;
  if constexpr (kBF16) asm("add.rn.f32.bf16 %0, %1, %2;" : "=f"(r) : "h"(a), "f"(c));
  else asm("add.rn.f32.f16 %0, %1, %2;" : "=f"(r) : "h"(a), "f"(c));
  return r;
}
template <bool kBF16>
__device__ __forceinline__ float sub_bits(uint16_t a, float c) {
  float r;
  if constexpr (kBF16) asm("sub.rn.f32.bf16 %0, %1, %2;" : "=f"(r) : "h"(a), "f"(c));
  else asm("sub.rn.f32.f16 %0, %1, %2;" : "=f"(r) : "h"(a), "f"(c));
  return r;
}
template <bool kBF16>
__device__ __forceinline__ RawMomentsGT<float> raw_moments_g_bits(const uint16_t (&h)[27]) {
  float z0[3][3], z1[3][3], z2[3][3];
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      const uint16_t a = h[slot(i, j, 0)], b = h[slot(i, j, 1)];
      const float c = bits_to_float<kBF16>(h[slot(i, j, 2)]);
      z2[i][j] = add_bits<kBF16>(a, c);
      z0[i][j] = add_bits<kBF16>(b, z2[i][j]);
      z1[i][j] = -sub_bits<kBF16>(a, c);
    }
  return raw_moments_from_z(z0, z1, z2);
}
#endif

// Density, velocity and D (second-order central moments less rho/3 I) of a cell.
template <typename T>
struct CellMomentsGT {
  T rho, inv_rho, ux, uy, uz;
  T dxx, dyy, dzz, dxy, dxz, dyz;
};
using CellMomentsG = CellMomentsGT<float>;

template <typename T>
PSL_HDI CellMomentsGT<T> cell_moments_from_raw(const RawMomentsGT<T>& r) {
  CellMomentsGT<T> m;
  m.rho = T(1.f) + r.rg;
  m.inv_rho = grecip(m.rho);
  m.ux = r.jx * m.inv_rho;
  m.uy = r.jy * m.inv_rho;
  m.uz = r.jz * m.inv_rho;
  const T r3 = r.rg * T(1.f / 3.f);
  m.dxx = gfma(-r.jx, m.ux, r.sxx - r3);
  m.dyy = gfma(-r.jy, m.uy, r.syy - r3);
  m.dzz = gfma(-r.jz, m.uz, r.szz - r3);
  m.dxy = gfma(-r.jx, m.uy, r.sxy);
  m.dxz = gfma(-r.jx, m.uz, r.sxz);
  m.dyz = gfma(-r.jy, m.uz, r.syz);
  return m;
}
template <typename T>
PSL_HDI CellMomentsGT<T> cell_moments_g(const T (&g)[27]) {
  return cell_moments_from_raw(raw_moments_g(g));
}

// Smagorinsky rate from D (include/cellFunctions.h:157-198): 1/tau without LES, else
// 1 / (tau/2 + sqrt(tau^2 + 18 C_s |Pi_neq| / rho)/2) with |Pi_neq| = |D|.
template <typename T>
PSL_HDI T smagorinsky_omega_g(const CellMomentsGT<T>& m, float omega0, float tau, float tau2, T cs18) {
  if (all_zero(cs18)) return T(omega0);
  const T p2 = gfma(m.dxx, m.dxx, gfma(m.dyy, m.dyy, m.dzz * m.dzz)) +
               T(2.f) * gfma(m.dxy, m.dxy, gfma(m.dxz, m.dxz, m.dyz * m.dyz));
  const T p = gsqrt(p2);
  const T w = grecip(gfma(T(0.5f), T(tau), T(0.5f) * gsqrt(gfma(cs18 * m.inv_rho, p, T(tau2)))));
  return sel_zero(cs18, T(omega0), w);
}

// One axis of the backward transform on pre-halved inputs (m1' = m1/2, m2' = m2/2), with
// hu2 = u^2/2, hu = u/2, tu = 2u: (m0, m1', m2') -> (f(-1), f(0), f(+1)).
template <typename T>
struct BwdAxis {
  T hu2, hu, tu;
  PSL_HDI explicit BwdAxis(T u) : hu2(T(0.5f) * u * u), hu(T(0.5f) * u), tu(T(2.f) * u) {}
};

template <typename T>
PSL_HDI void bwd_full(T& a, T& b, T& c, const BwdAxis<T>& k) {
  const T m0 = a, m1 = b, m2 = c;
  const T h = gfma(k.hu2, m0, gfma(k.tu, m1, m2));
  const T e = gfma(k.hu, m0, m1);
  a = h - e;
  b = gfma(T(-2.f), h, m0);
  c = h + e;
}
// m1' = 0
template <typename T>
PSL_HDI void bwd_even(T& a, T& b, T& c, const BwdAxis<T>& k) {
  const T m0 = a, m2 = c;
  const T h = gfma(k.hu2, m0, m2);
  const T e = k.hu * m0;
  a = h - e;
  b = gfma(T(-2.f), h, m0);
  c = h + e;
}
// m0 = m2' = 0: f(-1) = (2u - 1) m1', f(0) = -4u m1', f(+1) = (2u + 1) m1'
template <typename T>
PSL_HDI void bwd_odd(T& a, T& b, T& c, T cm, T c0, T cp) {
  const T m1 = b;
  a = cm * m1;
  b = c0 * m1;
  c = cp * m1;
}
// full triple, weights subtracted: (g(-1), g(0), g(+1)) = (f(-1) - wpm, f(0) - w0, f(+1) - wpm)
template <typename T>
PSL_HDI void bwd_full_w(T& a, T& b, T& c, const BwdAxis<T>& k, float wpm, float w0) {
  const T m0 = a, m1 = b, m2 = c;
  const T h = gfma(k.hu2, m0, gfma(k.tu, m1, m2)) - T(wpm);
  const T e = gfma(k.hu, m0, m1);
  a = h - e;
  b = gfma(T(-2.f), h, m0 - T(w0 + 2.f * wpm));
  c = h + e;
}

// Post-collision g' = f' - w from rho, u and the relaxed second-order central moments
// s** (first-order central moments zero, third-order cumulants zero; the fourth- and
// sixth-order central moments follow as in include/applyCollision.h:178-200).
template <typename T>
PSL_HDI void populations_g(T (&g)[27], T rho, T inv_rho, T ux, T uy, T uz, T s200, T s020, T s002, T s011, T s101,
                           T s110) {
  // pre-scaled inputs: K[i][j][k] * 2^-(number of non-zero orders)
  const T a200 = T(0.5f) * s200, a020 = T(0.5f) * s020, a002 = T(0.5f) * s002;
  const T a011 = T(0.25f) * s011, a101 = T(0.25f) * s101, a110 = T(0.25f) * s110;
  const T k211 = gfma(a200, a011, T(4.f) * a101 * a110) * inv_rho;
  const T k121 = gfma(a020, a101, T(4.f) * a110 * a011) * inv_rho;
  const T k112 = gfma(a002, a110, T(4.f) * a011 * a101) * inv_rho;
  const T k220 = gfma(a020, a200, T(8.f) * a110 * a110) * inv_rho;
  const T k022 = gfma(a002, a020, T(8.f) * a011 * a011) * inv_rho;
  const T k202 = gfma(a200, a002, T(8.f) * a101 * a101) * inv_rho;
  const T k222 =
      (a200 * k022 + a020 * k202 + a002 * k220 + T(16.f) * (a011 * k211 + a101 * k121 + a110 * k112)) * inv_rho -
      (T(128.f) * a110 * a101 * a011 + T(16.f) * (a101 * a101 * a020 + a011 * a011 * a200 + a110 * a110 * a002) +
       T(2.f) * a200 * a020 * a002) *
          (inv_rho * inv_rho);

  // G[x-slot][y-order][z-order] after the x pass
  T G[3][3][3];
  const BwdAxis<T> bx(ux), by(uy), bz(uz);
  const T xm = gfma(T(2.f), ux, T(-1.f)), x0 = T(-4.f) * ux, xp = gfma(T(2.f), ux, T(1.f));
  const T zero(0.f);
  G[0][0][0] = rho;  G[1][0][0] = zero; G[2][0][0] = a200;
  bwd_even(G[0][0][0], G[1][0][0], G[2][0][0], bx);
  G[0][0][1] = zero; G[1][0][1] = a101; G[2][0][1] = zero;
  bwd_odd(G[0][0][1], G[1][0][1], G[2][0][1], xm, x0, xp);
  G[0][0][2] = a002; G[1][0][2] = zero; G[2][0][2] = k202;
  bwd_even(G[0][0][2], G[1][0][2], G[2][0][2], bx);
  G[0][1][0] = zero; G[1][1][0] = a110; G[2][1][0] = zero;
  bwd_odd(G[0][1][0], G[1][1][0], G[2][1][0], xm, x0, xp);
  G[0][1][1] = a011; G[1][1][1] = zero; G[2][1][1] = k211;
  bwd_even(G[0][1][1], G[1][1][1], G[2][1][1], bx);
  G[0][1][2] = zero; G[1][1][2] = k112; G[2][1][2] = zero;
  bwd_odd(G[0][1][2], G[1][1][2], G[2][1][2], xm, x0, xp);
  G[0][2][0] = a020; G[1][2][0] = zero; G[2][2][0] = k220;
  bwd_even(G[0][2][0], G[1][2][0], G[2][2][0], bx);
  G[0][2][1] = zero; G[1][2][1] = k121; G[2][2][1] = zero;
  bwd_odd(G[0][2][1], G[1][2][1], G[2][2][1], xm, x0, xp);
  G[0][2][2] = k022; G[1][2][2] = zero; G[2][2][2] = k222;
  bwd_even(G[0][2][2], G[1][2][2], G[2][2][2], bx);
  // y pass
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int c = 0; c < 3; ++c) bwd_full(G[a][0][c], G[a][1][c], G[a][2][c], by);
  // z pass, weights subtracted
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = 0; b < 3; ++b) {
      T m0 = G[a][b][0], m1 = G[a][b][1], m2 = G[a][b][2];
      bwd_full_w(m0, m1, m2, bz, lattice_weight(slot(a, b, 0)), lattice_weight(slot(a, b, 1)));
      g[slot(a, b, 0)] = m0;
      g[slot(a, b, 1)] = m1;
      g[slot(a, b, 2)] = m2;
    }
}

// Relaxation at shear rate w (bulk at 1; include/applyCollision.h:119-200) from D, then
// the backward transform: g (post-streaming deviations) -> g' (post-collision).
template <typename T>
PSL_HDI void relax_rebuild_g(T (&g)[27], const CellMomentsGT<T>& m, T w) {
  const T rho = m.rho, inv_rho = m.inv_rho;
  const T hw = T(0.5f) * w * inv_rho;
  // c200 + c020 + c002 - rho = Dxx + Dyy + Dzz;  2 c200 - c020 - c002 = 2 Dxx - Dyy - Dzz
  const T dxu = -hw * (T(2.f) * m.dxx - m.dyy - m.dzz) - T(0.5f) * inv_rho * (m.dxx + m.dyy + m.dzz);
  const T dyv = gfma(T(3.f) * hw, m.dxx - m.dyy, dxu);
  const T dzw = gfma(T(3.f) * hw, m.dxx - m.dzz, dxu);
  const T om1 = T(1.f) - w;
  const T ux2 = m.ux * m.ux, uy2 = m.uy * m.uy, uz2 = m.uz * m.uz;
  const T gg = T(3.f) * rho * (T(1.f) - T(0.5f) * w);
  const T ea = om1 * (m.dxx - m.dyy) - gg * (ux2 * dxu - uy2 * dyv);
  const T eb = om1 * (m.dxx - m.dzz) - gg * (ux2 * dxu - uz2 * dzw);
  const T ec = rho - T(1.5f) * rho * (ux2 * dxu + uy2 * dyv + uz2 * dzw);
  const T s200 = T(1.f / 3.f) * (ea + eb + ec);
  const T s020 = T(1.f / 3.f) * (eb - T(2.f) * ea + ec);
  const T s002 = T(1.f / 3.f) * (ea - T(2.f) * eb + ec);
  populations_g(g, rho, inv_rho, m.ux, m.uy, m.uz, s200, s020, s002, om1 * m.dyz, om1 * m.dxz, om1 * m.dxy);
}

}  // namespace psl
