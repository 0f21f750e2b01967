// D3Q27 cumulant collision with Smagorinsky LES, and the refinement moment rescaling,
// written for registers: every loop is unrolled over compile-time indices, so the 27
// populations and 27 central moments never leave the register file.
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
//   * constants the reference writes as double literals (3.0 * omega ...) are float.
#pragma once
#include "psl_lattice.cuh"

namespace psl {

// ---- one axis of the central-moment transform (Geier 2015 eqs 43-45) ----------------------
// (f at slot -1, 0, +1) -> (moment of order 0, 1, 2 about u)
__device__ __forceinline__ void chimera_fwd(float& a, float& b, float& c, float u, float u2) {
  const float pm = c + a;
  const float sum = pm + b;
  const float diff = c - a;
  b = fmaf(-u, sum, diff);
  c = fmaf(u2, sum, fmaf(-2.f * u, diff, pm));
  a = sum;
}

// Per-velocity-component coefficients of the inverse transform (Geier 2015 eqs 88-96):
//   f(-1) = m0 (u^2-u)/2 + m1 (u - 1/2) + m2/2
//   f( 0) = m0 (1-u^2)   - m1 2u        - m2
//   f(+1) = m0 (u^2+u)/2 + m1 (u + 1/2) + m2/2
struct BwdCoef {
  float am, bm, a0, b0, ap, bp;
  __device__ __forceinline__ explicit BwdCoef(float u) {
    const float u2 = u * u;
    am = 0.5f * (u2 - u);
    bm = u - 0.5f;
    a0 = 1.f - u2;
    b0 = -2.f * u;
    ap = 0.5f * (u2 + u);
    bp = u + 0.5f;
  }
};

// Inverse transform of one triple; H0/H1/H2 say which input moments can be non-zero
// (the zero ones are compile-time absent, so no multiply by 0.f is ever issued).
template <bool H0, bool H1, bool H2>
__device__ __forceinline__ void chimera_bwd(float& m0, float& m1, float& m2, const BwdCoef& k) {
  float fm = 0.f, f0 = 0.f, fp = 0.f;
  if (H0) {
    fm = k.am * m0;
    f0 = k.a0 * m0;
    fp = k.ap * m0;
  }
  if (H1) {
    fm = H0 ? fmaf(k.bm, m1, fm) : k.bm * m1;
    f0 = H0 ? fmaf(k.b0, m1, f0) : k.b0 * m1;
    fp = H0 ? fmaf(k.bp, m1, fp) : k.bp * m1;
  }
  if (H2) {
    fm = (H0 || H1) ? fmaf(0.5f, m2, fm) : 0.5f * m2;
    f0 = (H0 || H1) ? f0 - m2 : -m2;
    fp = (H0 || H1) ? fmaf(0.5f, m2, fp) : 0.5f * m2;
  }
  m0 = fm;
  m1 = f0;
  m2 = fp;
}

// Forward transform of all 27 populations.  K[i][j][k] holds slots on entry and central
// moments (order i in x, j in y, k in z) on exit.  Also returns rho and u, accumulated
// from the z-line sums and differences of the first pass.
__device__ __forceinline__ void central_moments(const float (&f)[27], float (&K)[3][3][3], float& rho, float& ux,
                                                float& uy, float& uz, float& inv_rho) {
  float sum[3][3], diff[3][3], pm[3][3];
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      const float a = f[slot(i, j, 0)], b = f[slot(i, j, 1)], c = f[slot(i, j, 2)];
      pm[i][j] = c + a;
      sum[i][j] = pm[i][j] + b;
      diff[i][j] = c - a;
    }
  // rho, momentum from the line sums
  float sx[3], sy[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) sx[i] = (sum[i][0] + sum[i][2]) + sum[i][1];
#pragma unroll
  for (int j = 0; j < 3; ++j) sy[j] = (sum[0][j] + sum[2][j]) + sum[1][j];
  rho = (sx[0] + sx[2]) + sx[1];
  const float jx = sx[2] - sx[0];
  const float jy = sy[2] - sy[0];
  const float jz = ((diff[0][0] + diff[0][1]) + (diff[0][2] + diff[1][0])) +
                   ((diff[1][1] + diff[1][2]) + (diff[2][0] + diff[2][1])) + diff[2][2];
  inv_rho = 1.f / rho;
  ux = jx * inv_rho;
  uy = jy * inv_rho;
  uz = jz * inv_rho;
  const float uz2 = uz * uz, uy2 = uy * uy, ux2 = ux * ux;
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      K[i][j][0] = sum[i][j];
      K[i][j][1] = fmaf(-uz, sum[i][j], diff[i][j]);
      K[i][j][2] = fmaf(uz2, sum[i][j], fmaf(-2.f * uz, diff[i][j], pm[i][j]));
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

// Post-collision central moments (zero entries implicit) -> populations.
// Inputs: k000 (= rho), first-order moments (already negated), relaxed second-order
// cumulants s***, and inv_rho.  Higher central moments follow from the zero higher
// cumulants (Geier 2015 eqs 81, 82, 84; include/applyCollision.h:178-200).
__device__ __forceinline__ void populations_from_cumulants(float (&f)[27], float k000, float k100, float k010,
                                                           float k001, float s200, float s020, float s002,
                                                           float s011, float s101, float s110, float inv_rho,
                                                           float ux, float uy, float uz) {
  const float k211 = (s200 * s011 + 2.f * s101 * s110) * inv_rho;
  const float k121 = (s020 * s101 + 2.f * s110 * s011) * inv_rho;
  const float k112 = (s002 * s110 + 2.f * s011 * s101) * inv_rho;
  const float k220 = (s020 * s200 + 2.f * s110 * s110) * inv_rho;
  const float k022 = (s002 * s020 + 2.f * s011 * s011) * inv_rho;
  const float k202 = (s200 * s002 + 2.f * s101 * s101) * inv_rho;
  const float k222 = (s200 * k022 + s020 * k202 + s002 * k220 + 4.f * (s011 * k211 + s101 * k121 + s110 * k112)) * inv_rho -
                     (16.f * s110 * s101 * s011 + 4.f * (s101 * s101 * s020 + s011 * s011 * s200 + s110 * s110 * s002) +
                      2.f * s200 * s020 * s002) *
                         (inv_rho * inv_rho);

  // G[x-slot][y-order][z-order] after the x pass
  float G[3][3][3];
  const BwdCoef bx(ux), by(uy), bz(uz);
  // (y,z) orders: (0,0) full; (0,1) m0,m1; (0,2) m0,m2; (1,0) m0,m1; (1,1) m0,m2;
  // (1,2) m1; (2,0) m0,m2; (2,1) m1; (2,2) m0,m2
  G[0][0][0] = k000; G[1][0][0] = k100; G[2][0][0] = s200;
  chimera_bwd<true, true, true>(G[0][0][0], G[1][0][0], G[2][0][0], bx);
  G[0][0][1] = k001; G[1][0][1] = s101; G[2][0][1] = 0.f;
  chimera_bwd<true, true, false>(G[0][0][1], G[1][0][1], G[2][0][1], bx);
  G[0][0][2] = s002; G[1][0][2] = 0.f; G[2][0][2] = k202;
  chimera_bwd<true, false, true>(G[0][0][2], G[1][0][2], G[2][0][2], bx);
  G[0][1][0] = k010; G[1][1][0] = s110; G[2][1][0] = 0.f;
  chimera_bwd<true, true, false>(G[0][1][0], G[1][1][0], G[2][1][0], bx);
  G[0][1][1] = s011; G[1][1][1] = 0.f; G[2][1][1] = k211;
  chimera_bwd<true, false, true>(G[0][1][1], G[1][1][1], G[2][1][1], bx);
  G[0][1][2] = 0.f; G[1][1][2] = k112; G[2][1][2] = 0.f;
  chimera_bwd<false, true, false>(G[0][1][2], G[1][1][2], G[2][1][2], bx);
  G[0][2][0] = s020; G[1][2][0] = 0.f; G[2][2][0] = k220;
  chimera_bwd<true, false, true>(G[0][2][0], G[1][2][0], G[2][2][0], bx);
  G[0][2][1] = 0.f; G[1][2][1] = k121; G[2][2][1] = 0.f;
  chimera_bwd<false, true, false>(G[0][2][1], G[1][2][1], G[2][2][1], bx);
  G[0][2][2] = k022; G[1][2][2] = 0.f; G[2][2][2] = k222;
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
      float m0 = G[a][b][0], m1 = G[a][b][1], m2 = G[a][b][2];
      chimera_bwd<true, true, true>(m0, m1, m2, bz);
      f[slot(a, b, 0)] = m0;
      f[slot(a, b, 1)] = m1;
      f[slot(a, b, 2)] = m2;
    }
}

// Relaxation parameters of one grid: tau = 3 nu + 1/2; omega = 1/tau without LES.
struct Relaxation {
  float omega0;  // 1 / tau
  float tau;
  float tau2;    // tau^2
  float cs18;    // 18 * Smagorinsky constant (0 disables LES)
};

// Cumulant collision (include/applyCollision.h:6-295) with optional body force
// (half-force velocity shift of M40Impeller/applyCollisionCustomized.h:6-16).
template <bool kForce>
__device__ __forceinline__ void collide(float (&f)[27], const Relaxation& rx, float gx = 0.f, float gy = 0.f,
                                        float gz = 0.f) {
  float K[3][3][3];
  float rho, ux, uy, uz, inv_rho;
  if (!kForce) {
    central_moments(f, K, rho, ux, uy, uz, inv_rho);
  } else {
    // the forced velocity shifts the frame of the central moments
    float r0, u0, v0, w0, ir0;
    central_moments(f, K, r0, u0, v0, w0, ir0);  // only rho/u are used from this pass
    rho = r0;
    inv_rho = ir0;
    ux = (u0 * rho + 0.5f * gx) * inv_rho;
    uy = (v0 * rho + 0.5f * gy) * inv_rho;
    uz = (w0 * rho + 0.5f * gz) * inv_rho;
    // redo the transform about the shifted velocity
    float sum[3][3], diff[3][3], pm[3][3];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        const float a = f[slot(i, j, 0)], b = f[slot(i, j, 1)], c = f[slot(i, j, 2)];
        pm[i][j] = c + a;
        sum[i][j] = pm[i][j] + b;
        diff[i][j] = c - a;
      }
    const float uz2 = uz * uz, uy2 = uy * uy, ux2 = ux * ux;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        K[i][j][0] = sum[i][j];
        K[i][j][1] = fmaf(-uz, sum[i][j], diff[i][j]);
        K[i][j][2] = fmaf(uz2, sum[i][j], fmaf(-2.f * uz, diff[i][j], pm[i][j]));
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
  const float k000 = K[0][0][0], k100 = K[1][0][0], k010 = K[0][1][0], k001 = K[0][0][1];
  const float c200 = K[2][0][0], c020 = K[0][2][0], c002 = K[0][0][2];
  const float c011 = K[0][1][1], c101 = K[1][0][1], c110 = K[1][1][0];

  // Smagorinsky relaxation rate (include/cellFunctions.h:157-198)
  float w = rx.omega0;
  if (rx.cs18 != 0.f) {
    const float third = rho * (1.f / 3.f);
    const float pxx = c200 - third, pyy = c020 - third, pzz = c002 - third;
    const float p2 = pxx * pxx + pyy * pyy + pzz * pzz + 2.f * (c011 * c011 + c101 * c101 + c110 * c110);
    const float p = sqrtf(p2);
    const float tau_les = 0.5f * rx.tau + 0.5f * sqrtf(fmaf(rx.cs18 * inv_rho, p, rx.tau2));
    w = 1.f / tau_les;
  }

  // relaxation of the second-order cumulants (Geier 2015 eqs 55-65)
  const float hw = 0.5f * w * inv_rho;
  const float dxu = -hw * (2.f * c200 - c020 - c002) - 0.5f * inv_rho * (c200 + c020 + c002 - k000);
  const float dyv = fmaf(3.f * hw, c200 - c020, dxu);
  const float dzw = fmaf(3.f * hw, c200 - c002, dxu);
  const float om1 = 1.f - w;
  const float s110 = om1 * c110;
  const float s101 = om1 * c101;
  const float s011 = om1 * c011;
  const float ux2 = ux * ux, uy2 = uy * uy, uz2 = uz * uz;
  const float g = 3.f * rho * (1.f - 0.5f * w);
  const float ea = om1 * (c200 - c020) - g * (ux2 * dxu - uy2 * dyv);
  const float eb = om1 * (c200 - c002) - g * (ux2 * dxu - uz2 * dzw);
  const float ec = k000 - 1.5f * rho * (ux2 * dxu + uy2 * dyv + uz2 * dzw);
  const float s200 = (1.f / 3.f) * (ea + eb + ec);
  const float s020 = (1.f / 3.f) * (eb - 2.f * ea + ec);
  const float s002 = (1.f / 3.f) * (ea - 2.f * eb + ec);

  populations_from_cumulants(f, k000, -k100, -k010, -k001, s200, s020, s002, s011, s101, s110, inv_rho, ux, uy, uz);
}

// Moment rescaling across a 2:1 level change (include/gridRefinementFunctions.h:6-281).
__device__ __forceinline__ void rescale(float (&f)[27], bool coarse_to_fine) {
  float K[3][3][3];
  float rho, ux, uy, uz, inv_rho;
  central_moments(f, K, rho, ux, uy, uz, inv_rho);
  const float p200 = K[2][0][0], p020 = K[0][2][0], p002 = K[0][0][2];
  const float p011 = K[0][1][1], p101 = K[1][0][1], p110 = K[1][1][0];
  float c200, c020, c002, c011, c101, c110;
  if (coarse_to_fine) {
    c200 = (2.f / 3.f) * p200 + (1.f / 6.f) * p020 + (1.f / 6.f) * p002;
    c020 = (1.f / 6.f) * p200 + (2.f / 3.f) * p020 + (1.f / 6.f) * p002;
    c002 = (1.f / 6.f) * p200 + (1.f / 6.f) * p020 + (2.f / 3.f) * p002;
    c011 = 0.5f * p011;
    c101 = 0.5f * p101;
    c110 = 0.5f * p110;
  } else {
    c200 = (5.f / 3.f) * p200 - (1.f / 3.f) * p020 - (1.f / 3.f) * p002;
    c020 = -(1.f / 3.f) * p200 + (5.f / 3.f) * p020 - (1.f / 3.f) * p002;
    c002 = -(1.f / 3.f) * p200 - (1.f / 3.f) * p020 + (5.f / 3.f) * p002;
    c011 = 2.f * p011;
    c101 = 2.f * p101;
    c110 = 2.f * p110;
  }
  // rescaleF negates the first-order central moments too (gridRefinementFunctions.h:154-156)
  populations_from_cumulants(f, K[0][0][0], -K[1][0][0], -K[0][1][0], -K[0][0][1], c200, c020, c002, c011, c101, c110,
                             inv_rho, ux, uy, uz);
}

}  // namespace psl
