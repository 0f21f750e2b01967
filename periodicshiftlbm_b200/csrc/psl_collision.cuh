// D3Q27 cumulant collision with Smagorinsky LES, and the refinement moment rescaling,
// written for registers: every loop is unrolled over compile-time indices, so the 27
// populations and 27 central moments never leave the register file.  Templated on the
// arithmetic type: float for every production storage form, double only for the FP64
// oracle runs.
//
// Follows include/applyCollision.h:6-295 (Geier et al. 2015, "all-one" model: the six
// second-order cumulants are relaxed -- shear at omega_LES, bulk at 1 -- and every
// cumulant of order >= 3 is set to zero), include/cellFunctions.h:157-198 (Smagorinsky
// omega) and include/gridRefinementFunctions.h:6-281 (rescaleF).  Differences from the
// reference that change rounding only (results agree to FP32 rounding):
//   * density and momentum are accumulated along the z-lines of the transform;
//   * 1/rho is computed once and multiplied;
//   * |Pi_neq| for the Smagorinsky term is taken from the second-order central moments
//     (Pi_neq_aa = C_aa - rho/3, Pi_neq_ab = C_ab, exact for the D3Q27 second-order
//     equilibrium) instead of summing 27 explicit f - feq differences;
//   * constants the reference writes as double literals (3.0 * omega ...) are of type T.
#pragma once
#include "psl_lattice.cuh"

namespace psl {

__device__ __forceinline__ float fmat(float a, float b, float c) { return fmaf(a, b, c); }
__device__ __forceinline__ double fmat(double a, double b, double c) { return fma(a, b, c); }

// Scalar type of an arithmetic type (the lane type of a packed pair, see psl_pair.cuh).
template <typename T>
struct scalar_of {
  using type = T;
};
template <typename T>
using scalar_t = typename scalar_of<T>::type;

// ---- one axis of the central-moment transform (Geier 2015 eqs 43-45) ----------------------
// (f at slot -1, 0, +1) -> (moment of order 0, 1, 2 about u)
template <typename T>
__device__ __forceinline__ void chimera_fwd(T& a, T& b, T& c, T u, T u2) {
  const T pm = c + a;
  const T sum = pm + b;
  const T diff = c - a;
  b = fmat(-u, sum, diff);
  c = fmat(u2, sum, fmat(T(-2) * u, diff, pm));
  a = sum;
}

// Per-velocity-component coefficients of the inverse transform (Geier 2015 eqs 88-96):
//   f(-1) = m0 (u^2-u)/2 + m1 (u - 1/2) + m2/2
//   f( 0) = m0 (1-u^2)   - m1 2u        - m2
//   f(+1) = m0 (u^2+u)/2 + m1 (u + 1/2) + m2/2
template <typename T>
struct BwdCoef {
  T am, bm, a0, b0, ap, bp;
  __device__ __forceinline__ explicit BwdCoef(T u) {
    const T u2 = u * u;
    am = T(0.5) * (u2 - u);
    bm = u - T(0.5);
    a0 = T(1) - u2;
    b0 = T(-2) * u;
    ap = T(0.5) * (u2 + u);
    bp = u + T(0.5);
  }
};

// Inverse transform of one triple; H0/H1/H2 say which input moments can be non-zero
// (the zero ones are compile-time absent, so no multiply by zero is ever issued).
template <bool H0, bool H1, bool H2, typename T>
__device__ __forceinline__ void chimera_bwd(T& m0, T& m1, T& m2, const BwdCoef<T>& k) {
  T fm = T(0), f0 = T(0), fp = T(0);
  if (H0) {
    fm = k.am * m0;
    f0 = k.a0 * m0;
    fp = k.ap * m0;
  }
  if (H1) {
    fm = H0 ? fmat(k.bm, m1, fm) : k.bm * m1;
    f0 = H0 ? fmat(k.b0, m1, f0) : k.b0 * m1;
    fp = H0 ? fmat(k.bp, m1, fp) : k.bp * m1;
  }
  if (H2) {
    fm = (H0 || H1) ? fmat(T(0.5), m2, fm) : T(0.5) * m2;
    f0 = (H0 || H1) ? f0 - m2 : -m2;
    fp = (H0 || H1) ? fmat(T(0.5), m2, fp) : T(0.5) * m2;
  }
  m0 = fm;
  m1 = f0;
  m2 = fp;
}

template <typename T>
__device__ __forceinline__ void line_sums(const T (&f)[27], T (&sum)[3][3], T (&diff)[3][3], T (&pm)[3][3]) {
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      const T a = f[slot(i, j, 0)], b = f[slot(i, j, 1)], c = f[slot(i, j, 2)];
      pm[i][j] = c + a;
      sum[i][j] = pm[i][j] + b;
      diff[i][j] = c - a;
    }
}

// Central moments about (ux, uy, uz) from the z-line sums: K[i][j][k] = moment of order i
// in x, j in y, k in z.
template <typename T>
__device__ __forceinline__ void transform_about(const T (&sum)[3][3], const T (&diff)[3][3], const T (&pm)[3][3], T ux,
                                                T uy, T uz, T (&K)[3][3][3]) {
  const T uz2 = uz * uz, uy2 = uy * uy, ux2 = ux * ux;
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      K[i][j][0] = sum[i][j];
      K[i][j][1] = fmat(-uz, sum[i][j], diff[i][j]);
      K[i][j][2] = fmat(uz2, sum[i][j], fmat(T(-2) * uz, diff[i][j], pm[i][j]));
    }
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int k = 0; k < 3; ++k) chimera_fwd(K[i][0][k], K[i][1][k], K[i][2][k], uy, uy2);
#pragma unroll
  for (int j = 0; j < 3; ++j)
#pragma unroll
    for (int k = 0; k < 3; ++k) chimera_fwd(K[0][j][k], K[1][j][k], K[2][j][k], ux, ux2);
}

// Forward transform of all 27 populations, returning rho, u and 1/rho; rho and the
// momentum come from the z-line sums and differences of the first pass.
template <typename T>
__device__ __forceinline__ void central_moments(const T (&f)[27], T (&K)[3][3][3], T& rho, T& ux, T& uy, T& uz,
                                                T& inv_rho) {
  T sum[3][3], diff[3][3], pm[3][3];
  line_sums(f, sum, diff, pm);
  T sx[3], sy[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) sx[i] = (sum[i][0] + sum[i][2]) + sum[i][1];
#pragma unroll
  for (int j = 0; j < 3; ++j) sy[j] = (sum[0][j] + sum[2][j]) + sum[1][j];
  rho = (sx[0] + sx[2]) + sx[1];
  const T jx = sx[2] - sx[0];
  const T jy = sy[2] - sy[0];
  const T jz = ((diff[0][0] + diff[0][1]) + (diff[0][2] + diff[1][0])) +
               ((diff[1][1] + diff[1][2]) + (diff[2][0] + diff[2][1])) + diff[2][2];
  inv_rho = T(1) / rho;
  ux = jx * inv_rho;
  uy = jy * inv_rho;
  uz = jz * inv_rho;
  transform_about(sum, diff, pm, ux, uy, uz, K);
}

// Post-collision central moments (zero entries implicit) -> populations.
// Inputs: k000 (= rho), first-order moments (already negated), relaxed second-order
// cumulants s***, and inv_rho.  Higher central moments follow from the zero higher
// cumulants (Geier 2015 eqs 81, 82, 84; include/applyCollision.h:178-200).
template <typename T>
__device__ __forceinline__ void populations_from_cumulants(T (&f)[27], T k000, T k100, T k010, T k001, T s200, T s020,
                                                           T s002, T s011, T s101, T s110, T inv_rho, T ux, T uy, T uz) {
  const T k211 = (s200 * s011 + T(2) * s101 * s110) * inv_rho;
  const T k121 = (s020 * s101 + T(2) * s110 * s011) * inv_rho;
  const T k112 = (s002 * s110 + T(2) * s011 * s101) * inv_rho;
  const T k220 = (s020 * s200 + T(2) * s110 * s110) * inv_rho;
  const T k022 = (s002 * s020 + T(2) * s011 * s011) * inv_rho;
  const T k202 = (s200 * s002 + T(2) * s101 * s101) * inv_rho;
  const T k222 = (s200 * k022 + s020 * k202 + s002 * k220 + T(4) * (s011 * k211 + s101 * k121 + s110 * k112)) * inv_rho -
                 (T(16) * s110 * s101 * s011 + T(4) * (s101 * s101 * s020 + s011 * s011 * s200 + s110 * s110 * s002) +
                  T(2) * s200 * s020 * s002) *
                     (inv_rho * inv_rho);

  // G[x-slot][y-order][z-order] after the x pass
  T G[3][3][3];
  const BwdCoef<T> bx(ux), by(uy), bz(uz);
  // (y,z) orders: (0,0) full; (0,1) m0,m1; (0,2) m0,m2; (1,0) m0,m1; (1,1) m0,m2;
  // (1,2) m1; (2,0) m0,m2; (2,1) m1; (2,2) m0,m2
  G[0][0][0] = k000; G[1][0][0] = k100; G[2][0][0] = s200;
  chimera_bwd<true, true, true>(G[0][0][0], G[1][0][0], G[2][0][0], bx);
  G[0][0][1] = k001; G[1][0][1] = s101; G[2][0][1] = T(0);
  chimera_bwd<true, true, false>(G[0][0][1], G[1][0][1], G[2][0][1], bx);
  G[0][0][2] = s002; G[1][0][2] = T(0); G[2][0][2] = k202;
  chimera_bwd<true, false, true>(G[0][0][2], G[1][0][2], G[2][0][2], bx);
  G[0][1][0] = k010; G[1][1][0] = s110; G[2][1][0] = T(0);
  chimera_bwd<true, true, false>(G[0][1][0], G[1][1][0], G[2][1][0], bx);
  G[0][1][1] = s011; G[1][1][1] = T(0); G[2][1][1] = k211;
  chimera_bwd<true, false, true>(G[0][1][1], G[1][1][1], G[2][1][1], bx);
  G[0][1][2] = T(0); G[1][1][2] = k112; G[2][1][2] = T(0);
  chimera_bwd<false, true, false>(G[0][1][2], G[1][1][2], G[2][1][2], bx);
  G[0][2][0] = s020; G[1][2][0] = T(0); G[2][2][0] = k220;
  chimera_bwd<true, false, true>(G[0][2][0], G[1][2][0], G[2][2][0], bx);
  G[0][2][1] = T(0); G[1][2][1] = k121; G[2][2][1] = T(0);
  chimera_bwd<false, true, false>(G[0][2][1], G[1][2][1], G[2][2][1], bx);
  G[0][2][2] = k022; G[1][2][2] = T(0); G[2][2][2] = k222;
  chimera_bwd<true, false, true>(G[0][2][2], G[1][2][2], G[2][2][2], bx);
  // y pass (all inputs non-zero in general)
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int c = 0; c < 3; ++c) chimera_bwd<true, true, true>(G[a][0][c], G[a][1][c], G[a][2][c], by);
  // z pass straight into the populations
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = 0; b < 3; ++b) {
      T m0 = G[a][b][0], m1 = G[a][b][1], m2 = G[a][b][2];
      chimera_bwd<true, true, true>(m0, m1, m2, bz);
      f[slot(a, b, 0)] = m0;
      f[slot(a, b, 1)] = m1;
      f[slot(a, b, 2)] = m2;
    }
}

// Relaxation parameters of one grid: tau = 3 nu + 1/2; omega = 1/tau without LES.
template <typename T>
struct RelaxationT {
  T omega0;  // 1 / tau
  T tau;
  T tau2;    // tau^2
  T cs18;    // 18 * Smagorinsky constant (0 disables LES)
};
using Relaxation = RelaxationT<float>;

// Relaxation of the second-order cumulants at shear rate w (bulk at 1, higher cumulants
// to 0; Geier 2015 eqs 55-65, include/applyCollision.h:119-200) and the inverse transform.
template <typename T>
__device__ __forceinline__ void relax_rebuild(T (&f)[27], const T (&K)[3][3][3], T rho, T ux, T uy, T uz, T inv_rho,
                                              T w) {
  const T k000 = K[0][0][0], k100 = K[1][0][0], k010 = K[0][1][0], k001 = K[0][0][1];
  const T c200 = K[2][0][0], c020 = K[0][2][0], c002 = K[0][0][2];
  const T c011 = K[0][1][1], c101 = K[1][0][1], c110 = K[1][1][0];
  const T hw = T(0.5) * w * inv_rho;
  const T dxu = -hw * (T(2) * c200 - c020 - c002) - T(0.5) * inv_rho * (c200 + c020 + c002 - k000);
  const T dyv = fmat(T(3) * hw, c200 - c020, dxu);
  const T dzw = fmat(T(3) * hw, c200 - c002, dxu);
  const T om1 = T(1) - w;
  const T s110 = om1 * c110;
  const T s101 = om1 * c101;
  const T s011 = om1 * c011;
  const T ux2 = ux * ux, uy2 = uy * uy, uz2 = uz * uz;
  const T g = T(3) * rho * (T(1) - T(0.5) * w);
  const T ea = om1 * (c200 - c020) - g * (ux2 * dxu - uy2 * dyv);
  const T eb = om1 * (c200 - c002) - g * (ux2 * dxu - uz2 * dzw);
  const T ec = k000 - T(1.5) * rho * (ux2 * dxu + uy2 * dyv + uz2 * dzw);
  const T s200 = T(scalar_t<T>(1) / scalar_t<T>(3)) * (ea + eb + ec);
  const T s020 = T(scalar_t<T>(1) / scalar_t<T>(3)) * (eb - T(2) * ea + ec);
  const T s002 = T(scalar_t<T>(1) / scalar_t<T>(3)) * (ea - T(2) * eb + ec);

  populations_from_cumulants(f, k000, -k100, -k010, -k001, s200, s020, s002, s011, s101, s110, inv_rho, ux, uy, uz);
}

// Smagorinsky relaxation rate (include/cellFunctions.h:157-198): 1/tau without LES, else
// 1/tau_LES with tau_LES = tau/2 + sqrt(tau^2 + 18 C_s |Pi_neq| / rho)/2, |Pi_neq| from the
// second-order central moments.
template <typename T>
__device__ __forceinline__ T smagorinsky_omega(const T (&K)[3][3][3], T rho, T inv_rho, const RelaxationT<scalar_t<T>>& rx) {
  T w = T(rx.omega0);
  if (rx.cs18 != scalar_t<T>(0)) {
    const T c200 = K[2][0][0], c020 = K[0][2][0], c002 = K[0][0][2];
    const T c011 = K[0][1][1], c101 = K[1][0][1], c110 = K[1][1][0];
    const T third = rho * T(scalar_t<T>(1) / scalar_t<T>(3));
    const T pxx = c200 - third, pyy = c020 - third, pzz = c002 - third;
    const T p2 = pxx * pxx + pyy * pyy + pzz * pzz + T(2) * (c011 * c011 + c101 * c101 + c110 * c110);
    const T p = sqrt(p2);
    const T tau_les = T(scalar_t<T>(0.5) * rx.tau) + T(0.5) * sqrt(fmat(T(rx.cs18) * inv_rho, p, T(rx.tau2)));
    w = T(1) / tau_les;
  }
  return w;
}

// Cumulant collision (include/applyCollision.h:6-295) with optional body force
// (half-force velocity shift of M40Impeller/applyCollisionCustomized.h:6-16).
// Returns the density.
template <bool kForce, typename T>
__device__ __forceinline__ T collide(T (&f)[27], const RelaxationT<scalar_t<T>>& rx, T gx = T(0), T gy = T(0),
                                     T gz = T(0)) {
  T K[3][3][3];
  T rho, ux, uy, uz, inv_rho;
  if (!kForce) {
    central_moments(f, K, rho, ux, uy, uz, inv_rho);
  } else {
    T sum[3][3], diff[3][3], pm[3][3];
    line_sums(f, sum, diff, pm);
    T sx[3], sy[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) sx[i] = (sum[i][0] + sum[i][2]) + sum[i][1];
#pragma unroll
    for (int j = 0; j < 3; ++j) sy[j] = (sum[0][j] + sum[2][j]) + sum[1][j];
    rho = (sx[0] + sx[2]) + sx[1];
    const T jz = ((diff[0][0] + diff[0][1]) + (diff[0][2] + diff[1][0])) +
                 ((diff[1][1] + diff[1][2]) + (diff[2][0] + diff[2][1])) + diff[2][2];
    inv_rho = T(1) / rho;
    // the forced velocity shifts the frame of the central moments
    ux = (sx[2] - sx[0] + T(0.5) * gx) * inv_rho;
    uy = (sy[2] - sy[0] + T(0.5) * gy) * inv_rho;
    uz = (jz + T(0.5) * gz) * inv_rho;
    transform_about(sum, diff, pm, ux, uy, uz, K);
  }
  relax_rebuild(f, K, rho, ux, uy, uz, inv_rho, smagorinsky_omega(K, rho, inv_rho, rx));
  return rho;
}

// Moment rescaling across a 2:1 level change (include/gridRefinementFunctions.h:6-281).
template <typename T>
__device__ __forceinline__ void rescale(T (&f)[27], bool coarse_to_fine) {
  T K[3][3][3];
  T rho, ux, uy, uz, inv_rho;
  central_moments(f, K, rho, ux, uy, uz, inv_rho);
  const T p200 = K[2][0][0], p020 = K[0][2][0], p002 = K[0][0][2];
  const T p011 = K[0][1][1], p101 = K[1][0][1], p110 = K[1][1][0];
  T c200, c020, c002, c011, c101, c110;
  if (coarse_to_fine) {
    c200 = T(scalar_t<T>(2) / scalar_t<T>(3)) * p200 + T(scalar_t<T>(1) / scalar_t<T>(6)) * p020 + T(scalar_t<T>(1) / scalar_t<T>(6)) * p002;
    c020 = T(scalar_t<T>(1) / scalar_t<T>(6)) * p200 + T(scalar_t<T>(2) / scalar_t<T>(3)) * p020 + T(scalar_t<T>(1) / scalar_t<T>(6)) * p002;
    c002 = T(scalar_t<T>(1) / scalar_t<T>(6)) * p200 + T(scalar_t<T>(1) / scalar_t<T>(6)) * p020 + T(scalar_t<T>(2) / scalar_t<T>(3)) * p002;
    c011 = T(0.5) * p011;
    c101 = T(0.5) * p101;
    c110 = T(0.5) * p110;
  } else {
    c200 = T(scalar_t<T>(5) / scalar_t<T>(3)) * p200 - T(scalar_t<T>(1) / scalar_t<T>(3)) * p020 - T(scalar_t<T>(1) / scalar_t<T>(3)) * p002;
    c020 = -T(scalar_t<T>(1) / scalar_t<T>(3)) * p200 + T(scalar_t<T>(5) / scalar_t<T>(3)) * p020 - T(scalar_t<T>(1) / scalar_t<T>(3)) * p002;
    c002 = -T(scalar_t<T>(1) / scalar_t<T>(3)) * p200 - T(scalar_t<T>(1) / scalar_t<T>(3)) * p020 + T(scalar_t<T>(5) / scalar_t<T>(3)) * p002;
    c011 = T(2) * p011;
    c101 = T(2) * p101;
    c110 = T(2) * p110;
  }
  // rescaleF negates the first-order central moments too (gridRefinementFunctions.h:154-156)
  populations_from_cumulants(f, K[0][0][0], -K[1][0][0], -K[0][1][0], -K[0][0][1], c200, c020, c002, c011, c101, c110,
                             inv_rho, ux, uy, uz);
}

}  // namespace psl
