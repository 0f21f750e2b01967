// CPU oracle: restatement of the reference's per-step lattice update (see psl_oracle.h).
//
// ORACLE / TEST INFRASTRUCTURE ONLY.  Loops over plain arrays, OpenMP over cells; the
// boundary conditions are evaluated from the coefficient tables in
// bc_oracle_generated.h (generic loops), independently of the straight-line CUDA code.

#include "psl_oracle.h"

#include <cmath>
#include <cstring>
#include <memory>

#include "bc_oracle_generated.h"
#include "psl_case_noise.h"

namespace oracle {

// index of velocity (x, y, z) in {-1,0,1}^3
static int qOf(int x, int y, int z) {
  for (int q = 0; q < 27; ++q)
    if (CX[q] == x && CY[q] == y && CZ[q] == z) return q;
  return -1;
}
static int opposite(int q) { return qOf(-CX[q], -CY[q], -CZ[q]); }

// ------------------------------------------------------------------------------------------
// Cell functions
// ------------------------------------------------------------------------------------------

// Second-order equilibrium, include/cellFunctions.h:60-121.
template <typename T>
void feq(T rho, T ux, T uy, T uz, T* out) {
  const T u2 = ux * ux + uy * uy + uz * uz;
  for (int q = 0; q < 27; ++q) {
    const T cu = T(CX[q]) * ux + T(CY[q]) * uy + T(CZ[q]) * uz;
    out[q] = rho * Weights<T>::w(q) * (T(1) + T(3) * cu + T(4.5) * cu * cu - T(1.5) * u2);
  }
}

// Density and velocity, include/cellFunctions.h:135-155.
template <typename T>
void rhoU(const T* f, T& rho, T& ux, T& uy, T& uz) {
  T r = 0, jx = 0, jy = 0, jz = 0;
  for (int q = 0; q < 27; ++q) {
    r += f[q];
    jx += T(CX[q]) * f[q];
    jy += T(CY[q]) * f[q];
    jz += T(CZ[q]) * f[q];
  }
  rho = r;
  ux = jx / r;
  uy = jy / r;
  uz = jz / r;
}

// Smagorinsky relaxation rate, include/cellFunctions.h:157-198: tau = 3 nu + 1/2 and
// tau_LES = tau/2 + sqrt(tau^2 + 18 Cs |Pi_neq| / rho)/2 with Pi_neq the second moments of
// f - feq.
template <typename T>
T omegaLES(const T* f, T rho, T ux, T uy, T uz, T nu, T cs) {
  const T tau = T(3) * nu + T(0.5);
  if (cs == T(0)) return T(1) / tau;
  T fe[27];
  feq(rho, ux, uy, uz, fe);
  T pi[3][3] = {};
  for (int q = 0; q < 27; ++q) {
    const T d = f[q] - fe[q];
    const int c[3] = {CX[q], CY[q], CZ[q]};
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b) pi[a][b] += T(c[a] * c[b]) * d;
  }
  T p = 0;
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) p += pi[a][b] * pi[a][b];
  p = std::sqrt(p);
  const T tauLES = T(0.5) * tau + T(0.5) * std::sqrt(tau * tau + T(18) * cs * (T(1) / rho) * p);
  return T(1) / tauLES;
}

// One axis of the central-moment ("chimera") transform, Geier et al. 2015 eqs 43-45:
// (f-, f0, f+) at velocity slots -1, 0, +1  ->  moments of order 0, 1, 2 about u.
template <typename T>
inline void chimeraForward(T& a, T& b, T& c, T u) {
  const T sum = (c + a) + b;
  const T diff = c - a;
  const T m1 = diff - u * sum;
  const T m2 = (c + a) - T(2) * u * diff + u * u * sum;
  a = sum;
  b = m1;
  c = m2;
}
// Inverse of chimeraForward, Geier et al. 2015 eqs 88-96.
template <typename T>
inline void chimeraBackward(T& m0, T& m1, T& m2, T u) {
  const T fm = (m0 * (u * u - u) + m1 * (T(2) * u - T(1)) + m2) * T(0.5);
  const T f0 = m0 * (T(1) - u * u) - T(2) * u * m1 - m2;
  const T fp = (m0 * (u * u + u) + m1 * (T(2) * u + T(1)) + m2) * T(0.5);
  m0 = fm;
  m1 = f0;
  m2 = fp;
}

// K[i][j][k]: axis slots (-1,0,+1 -> 0,1,2) before the transform, moment orders after.
template <typename T>
void toCentralMoments(const T* f, T ux, T uy, T uz, T K[3][3][3]) {
  for (int q = 0; q < 27; ++q) K[CX[q] + 1][CY[q] + 1][CZ[q] + 1] = f[q];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) chimeraForward(K[i][j][0], K[i][j][1], K[i][j][2], uz);
  for (int i = 0; i < 3; ++i)
    for (int k = 0; k < 3; ++k) chimeraForward(K[i][0][k], K[i][1][k], K[i][2][k], uy);
  for (int j = 0; j < 3; ++j)
    for (int k = 0; k < 3; ++k) chimeraForward(K[0][j][k], K[1][j][k], K[2][j][k], ux);
}

template <typename T>
void fromCentralMoments(T K[3][3][3], T ux, T uy, T uz, T* f) {
  for (int j = 0; j < 3; ++j)
    for (int k = 0; k < 3; ++k) chimeraBackward(K[0][j][k], K[1][j][k], K[2][j][k], ux);
  for (int i = 0; i < 3; ++i)
    for (int k = 0; k < 3; ++k) chimeraBackward(K[i][0][k], K[i][1][k], K[i][2][k], uy);
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) chimeraBackward(K[i][j][0], K[i][j][1], K[i][j][2], uz);
  for (int q = 0; q < 27; ++q) f[q] = K[CX[q] + 1][CY[q] + 1][CZ[q] + 1];
}

// Post-collision central moments from the relaxed second-order cumulants with every
// cumulant of order >= 3 set to zero ("all-one" cumulant model): Geier et al. 2015 eqs
// 81, 82, 84 (include/applyCollision.h:178-200), first-order moments negated (eqs 85-87).
template <typename T>
void cumulantsToCentralMoments(T rho, T k000, T k100, T k010, T k001, T c200, T c020, T c002, T c011, T c101,
                               T c110, T K[3][3][3]) {
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j)
      for (int k = 0; k < 3; ++k) K[i][j][k] = T(0);
  K[0][0][0] = k000;
  K[1][0][0] = -k100;
  K[0][1][0] = -k010;
  K[0][0][1] = -k001;
  K[2][0][0] = c200;
  K[0][2][0] = c020;
  K[0][0][2] = c002;
  K[0][1][1] = c011;
  K[1][0][1] = c101;
  K[1][1][0] = c110;
  K[2][1][1] = (c200 * c011 + T(2) * c101 * c110) / rho;
  K[1][2][1] = (c020 * c101 + T(2) * c110 * c011) / rho;
  K[1][1][2] = (c002 * c110 + T(2) * c011 * c101) / rho;
  K[2][2][0] = (c020 * c200 + T(2) * c110 * c110) / rho;
  K[0][2][2] = (c002 * c020 + T(2) * c011 * c011) / rho;
  K[2][0][2] = (c200 * c002 + T(2) * c101 * c101) / rho;
  K[2][2][2] = (c200 * K[0][2][2] + c020 * K[2][0][2] + c002 * K[2][2][0] +
                T(4) * (c011 * K[2][1][1] + c101 * K[1][2][1] + c110 * K[1][1][2])) / rho -
               (T(16) * c110 * c101 * c011 + T(4) * (c101 * c101 * c020 + c011 * c011 * c200 + c110 * c110 * c002) +
                T(2) * c200 * c020 * c002) / rho / rho;
}

// Cumulant collision with Smagorinsky LES, include/applyCollision.h:6-295.
// gx, gy, gz: optional body force (half-force velocity shift,
// M40Impeller/applyCollisionCustomized.h:6-16); zero for the plain update.
template <typename T>
void collide(T* f, T nu, T cs, T gx = 0, T gy = 0, T gz = 0) {
  T rho, ux, uy, uz;
  rhoU(f, rho, ux, uy, uz);
  if (gx != T(0) || gy != T(0) || gz != T(0)) {
    ux = ((ux * rho) + gx / T(2)) / rho;
    uy = ((uy * rho) + gy / T(2)) / rho;
    uz = ((uz * rho) + gz / T(2)) / rho;
  }
  T K[3][3][3];
  toCentralMoments(f, ux, uy, uz, K);
  const T k000 = K[0][0][0], k100 = K[1][0][0], k010 = K[0][1][0], k001 = K[0][0][1];
  const T c200 = K[2][0][0], c020 = K[0][2][0], c002 = K[0][0][2];
  const T c011 = K[0][1][1], c101 = K[1][0][1], c110 = K[1][1][0];
  const T w = omegaLES(f, rho, ux, uy, uz, nu, cs);

  // Geier 2015 eqs 58-60: velocity-derivative estimates
  const T dxu = -w * T(0.5) / rho * (T(2) * c200 - c020 - c002) - T(0.5) / rho * (c200 + c020 + c002 - k000);
  const T dyv = dxu + T(3) * w * T(0.5) / rho * (c200 - c020);
  const T dzw = dxu + T(3) * w * T(0.5) / rho * (c200 - c002);
  // eqs 55-57: off-diagonal second-order cumulants
  const T s110 = (T(1) - w) * c110;
  const T s101 = (T(1) - w) * c101;
  const T s011 = (T(1) - w) * c011;
  // eqs 61-65: diagonal second-order cumulants (bulk viscosity relaxed at rate 1)
  const T a = (T(1) - w) * (c200 - c020) - T(3) * rho * (T(1) - w * T(0.5)) * (ux * ux * dxu - uy * uy * dyv);
  const T b = (T(1) - w) * (c200 - c002) - T(3) * rho * (T(1) - w * T(0.5)) * (ux * ux * dxu - uz * uz * dzw);
  const T c = k000 - T(3) * rho * T(0.5) * (ux * ux * dxu + uy * uy * dyv + uz * uz * dzw);
  const T s200 = T(1) / T(3) * (a + b + c);
  const T s020 = T(1) / T(3) * (b - T(2) * a + c);
  const T s002 = T(1) / T(3) * (a - T(2) * b + c);

  cumulantsToCentralMoments(rho, k000, k100, k010, k001, s200, s020, s002, s011, s101, s110, K);
  fromCentralMoments(K, ux, uy, uz, f);
}

// Moment rescaling between refinement levels, include/gridRefinementFunctions.h:6-281:
// second-order central moments mapped by the coarse->fine (2/3,1/6,1/6; 1/2) or
// fine->coarse (5/3,-1/3,-1/3; 2) factors, higher cumulants zero, no relaxation.
template <typename T>
void rescale(T* f, bool coarseToFine) {
  T rho, ux, uy, uz;
  rhoU(f, rho, ux, uy, uz);
  T K[3][3][3];
  toCentralMoments(f, ux, uy, uz, K);
  const T p200 = K[2][0][0], p020 = K[0][2][0], p002 = K[0][0][2];
  const T p011 = K[0][1][1], p101 = K[1][0][1], p110 = K[1][1][0];
  T c200, c020, c002, c011, c101, c110;
  if (coarseToFine) {
    c200 = (T(2) / T(3)) * p200 + (T(1) / T(6)) * p020 + (T(1) / T(6)) * p002;
    c020 = (T(1) / T(6)) * p200 + (T(2) / T(3)) * p020 + (T(1) / T(6)) * p002;
    c002 = (T(1) / T(6)) * p200 + (T(1) / T(6)) * p020 + (T(2) / T(3)) * p002;
    c011 = T(0.5) * p011;
    c101 = T(0.5) * p101;
    c110 = T(0.5) * p110;
  } else {
    c200 = (T(5) / T(3)) * p200 - (T(1) / T(3)) * p020 - (T(1) / T(3)) * p002;
    c020 = -(T(1) / T(3)) * p200 + (T(5) / T(3)) * p020 - (T(1) / T(3)) * p002;
    c002 = -(T(1) / T(3)) * p200 - (T(1) / T(3)) * p020 + (T(5) / T(3)) * p002;
    c011 = T(2) * p011;
    c101 = T(2) * p101;
    c110 = T(2) * p110;
  }
  cumulantsToCentralMoments(rho, K[0][0][0], K[1][0][0], K[0][1][0], K[0][0][1], c200, c020, c002, c011, c101, c110, K);
  fromCentralMoments(K, ux, uy, uz, f);
}

// ------------------------------------------------------------------------------------------
// Boundary conditions (include/boundaryConditions/*.h) from the generated tables
// ------------------------------------------------------------------------------------------
inline int normalIndex(int nx, int ny, int nz) { return (nx + 1) * 9 + (ny + 1) * 3 + (nz + 1); }

// Imposed equilibrium moment m (helperMain.py:29-52 table, generated coefficients).
template <typename T>
T eqMoment(int m, T rho, T ux, T uy, T uz) {
  const oracle_bc::MeqPoly& p = oracle_bc::kMeq[m];
  T s = 0;
  for (int t = 0; t < p.n; ++t) {
    T v = T(p.t[t].coef);
    for (int r = 0; r < p.t[t].px; ++r) v *= ux;
    for (int r = 0; r < p.t[t].py; ++r) v *= uy;
    for (int r = 0; r < p.t[t].pz; ++r) v *= uz;
    s += v;
  }
  return rho * s;
}

template <typename T>
void mbbc(int normal, T* f, T rho, T ux, T uy, T uz) {  // applyMBBC.h
  const oracle_bc::NormalTable& t = oracle_bc::kNormals[normal];
  if (!t.valid) return;
  T s[19];
  for (int r = 0; r < t.n_unknown; ++r) {
    T known = 0;
    for (int q = 0; q < 27; ++q) known += T(t.mbbc_known[r][q]) * f[q];
    s[r] = eqMoment(t.mbbc_moment[r], rho, ux, uy, uz) - known;
  }
  for (int i = 0; i < t.n_unknown; ++i) {
    T v = 0;
    for (int r = 0; r < t.n_unknown; ++r) v += T(t.mbbc_inv[i][r]) * s[r];
    f[t.unknown[i]] = v;
  }
}

template <typename T>
void restoreRhoU(int normal, const T* f, T& rho, T& ux, T& uy, T& uz) {  // restoreRhoUxUyUz.h
  const oracle_bc::NormalTable& t = oracle_bc::kNormals[normal];
  if (!t.valid) return;
  T qv[4];
  for (int r = 0; r < 4; ++r) {
    qv[r] = 0;
    for (int q = 0; q < 27; ++q) qv[r] += T(t.rhou[r][q]) * f[q];
  }
  rho = qv[0];
  ux = qv[1] / rho;
  uy = qv[2] / rho;
  uz = qv[3] / rho;
}

template <typename T>
void restoreU(int normal, const T* f, T rho, T& ux, T& uy, T& uz) {  // restoreUxUyUz.h
  const oracle_bc::NormalTable& t = oracle_bc::kNormals[normal];
  if (!t.valid) return;
  T s[3];
  for (int r = 0; r < 3; ++r) {
    T v = 0;
    for (int q = 0; q < 27; ++q) v += T(t.u_known[r][q]) * f[q];
    s[r] = v / rho - T(t.u_rho[r]);
  }
  T u[3];
  for (int a = 0; a < 3; ++a) u[a] = T(t.u_inv[a][0]) * s[0] + T(t.u_inv[a][1]) * s[1] + T(t.u_inv[a][2]) * s[2];
  ux = u[0];
  uy = u[1];
  uz = u[2];
}

template <typename T>
void restoreRho(int normal, const T* f, T& rho, T ux, T uy, T uz) {  // restoreRho.h
  const oracle_bc::NormalTable& t = oracle_bc::kNormals[normal];
  if (!t.valid) return;
  T num = 0;
  for (int q = 0; q < 27; ++q) num += T(t.r_known[q]) * f[q];
  const T den = T(t.r_rho) + (T(t.r_u[0]) * ux + T(t.r_u[1]) * uy + T(t.r_u[2]) * uz);
  rho = num / den;
}

template <typename T>
void mirror(int normal, T* f) {  // results/applyMirror.h
  const oracle_bc::NormalTable& t = oracle_bc::kNormals[normal];
  if (!t.valid) return;
  T src[27];
  for (int q = 0; q < 27; ++q) src[q] = f[q];
  for (int q = 0; q < 27; ++q)
    if (t.mirror_src[q] >= 0) f[q] = src[t.mirror_src[q]];
}

template <typename T>
void bounceback(T* f) {  // applyBounceback.h:8-27
  T g[27];
  for (int q = 0; q < 27; ++q) g[q] = f[opposite(q)];
  for (int q = 0; q < 27; ++q) f[q] = g[q];
}

// applyMovingBounceback.h:8-60: f_q <- f_opp(q) + 6 w_q (c_q . u_w) for each pair.
template <typename T>
void movingBounceback(T* f, T ux, T uy, T uz) {
  T g[27];
  for (int q = 0; q < 27; ++q) {
    const int o = opposite(q);
    const T cu = T(CX[q]) * ux + T(CY[q]) * uy + T(CZ[q]) * uz;
    g[q] = f[o] + T(6) * Weights<T>::w(q) * cu;
  }
  for (int q = 0; q < 27; ++q) f[q] = g[q];
}

// ------------------------------------------------------------------------------------------
// Grids, markers and the per-step update
// ------------------------------------------------------------------------------------------
struct Info {
  int level = 0;
  float res = 1.f, ox = 0.f, oy = 0.f, oz = 0.f;
  float nu = 0.f;
  int nx = 0, ny = 0, nz = 0;
  long long n = 0;
  int iS = 0, jS = 0, kS = 0, iE = 0, jE = 0, kE = 0;  // refinement block (coarse side)
};

enum class Kind { Skip, Fluid, Solid, GivenU, GivenRho, Mirror };

template <typename T>
struct Grid {
  Info info;
  std::vector<T> f;   // [27][n], shifted (periodic-shift) addresses
  long long shift[27] = {};
  T* pop(int q) { return f.data() + (size_t)q * (size_t)info.n; }
  long long addr(int q, long long cell) const {
    long long a = cell + shift[q];
    if (a >= info.n) a -= info.n;
    return a;
  }
};

template <typename T>
struct Sim {
  CaseConfig cfg;
  std::vector<Grid<T>> grids;
};

// Marker hook for the sphere cases (oracle/ref_cases.cpp getMarkers, after
// flowAroundSphere/flowAroundSphereMainSingle.cu:41-67).
static Kind cellKind(const CaseConfig& c, const Info& I, int i, int j, int k) {
  const float x = i * I.res + I.ox, y = j * I.res + I.oy, z = k * I.res + I.oz;
  const float r2 = (x - c.sphereX) * (x - c.sphereX) + (y - c.sphereY) * (y - c.sphereY) + (z - c.sphereZ) * (z - c.sphereZ);
  if (r2 <= c.sphereR * c.sphereR) return Kind::Solid;
  if (I.level != 0) {
    if (i == 0 || i == I.nx - 1 || j == 0 || j == I.ny - 1 || k == 0 || k == I.nz - 1) return Kind::Skip;
    return Kind::Fluid;
  }
  const bool wall = (j == 0 || j == I.ny - 1 || k == 0 || k == I.nz - 1);
  if (c.wallMode == 1) {
    if (wall || i == 0) return Kind::GivenU;
    if (i == I.nx - 1) return Kind::GivenRho;
    return Kind::Fluid;
  }
  if (i == 0) return Kind::GivenU;
  if (i == I.nx - 1) return Kind::GivenRho;
  if (wall) return Kind::Mirror;
  return Kind::Fluid;
}

static int outerNormal(const Info& I, int i, int j, int k) {  // cellFunctions.h:46-58
  const int nx = (i == 0) ? -1 : (i == I.nx - 1 ? 1 : 0);
  const int ny = (j == 0) ? -1 : (j == I.ny - 1 ? 1 : 0);
  const int nz = (k == 0) ? -1 : (k == I.nz - 1 ? 1 : 0);
  return normalIndex(nx, ny, nz);
}

// applyStreaming.h:11-31: shift_q <- shift_q - (cx + Nx cy + Nx Ny cz), kept in [0, N).
static void streamShifts(long long* shift, const Info& I) {
  for (int q = 0; q < 27; ++q) {
    long long s = shift[q] - (CX[q] + (long long)I.nx * CY[q] + (long long)I.nx * I.ny * CZ[q]);
    while (s < 0) s += I.n;
    while (s >= I.n) s -= I.n;
    shift[q] = s;
  }
}

// applyLocalCellUpdate.h:1-74 (plus the free-slip customisation of oracle/ref_cases.cpp).
template <typename T>
static void localUpdate(Sim<T>& sim, Grid<T>& g) {
  const Info& I = g.info;
  const CaseConfig& c = sim.cfg;
  const T nu = T(I.nu);
  const T rhoGiven = T(1), uxGiven = T(c.uIn), uyGiven = T(0), uzGiven = T(0);
#pragma omp parallel for schedule(static)
  for (long long cell = 0; cell < I.n; ++cell) {
    const int i = (int)(cell % I.nx), j = (int)((cell / I.nx) % I.ny), k = (int)(cell / ((long long)I.nx * I.ny));
    const Kind kind = cellKind(c, I, i, j, k);
    if (kind == Kind::Skip) continue;
    if (i > I.iS + 1 && i < I.iE - 2 && j > I.jS + 1 && j < I.jE - 2 && k > I.kS + 1 && k < I.kE - 2) continue;
    T f[27];
    long long a[27];
    for (int q = 0; q < 27; ++q) {
      a[q] = g.addr(q, cell);
      f[q] = g.f[(size_t)q * I.n + a[q]];
    }
    if (kind == Kind::Solid) {
      bounceback(f);
    } else {
      if (kind != Kind::Fluid) {
        const int n = outerNormal(I, i, j, k);
        T rho = rhoGiven, ux = uxGiven, uy = uyGiven, uz = uzGiven;
        if (kind == Kind::Mirror) {
          mirror(n, f);
        } else {
          if (kind == Kind::GivenRho) restoreU(n, f, rho, ux, uy, uz);
          else if (kind == Kind::GivenU) restoreRho(n, f, rho, ux, uy, uz);
          mbbc(n, f, rho, ux, uy, uz);
        }
      }
      collide(f, nu, T(smagorinskyConstant(c, I.level, I.nx, i)));
    }
    for (int q = 0; q < 27; ++q) g.f[(size_t)q * I.n + a[q]] = f[q];
  }
}

template <typename T>
static void readCell(Grid<T>& g, long long cell, T* f) {
  for (int q = 0; q < 27; ++q) f[q] = g.f[(size_t)q * g.info.n + g.addr(q, cell)];
}
template <typename T>
static void writeCell(Grid<T>& g, long long cell, const T* f) {
  for (int q = 0; q < 27; ++q) g.f[(size_t)q * g.info.n + g.addr(q, cell)] = f[q];
}
static long long cellIndex(const Info& I, int i, int j, int k) {
  return ((long long)k * I.ny + j) * I.nx + i;
}

// gridRefinementFunctions.h:283-336: average of the 8 fine cells, rescaled fine->coarse,
// written to coarse cells of the box [b0, b1).
template <typename T>
static void restrictBox(Grid<T>& gc, Grid<T>& gf, const int b0[3], const int b1[3]) {
  const Info& C = gc.info;
  for (int k = b0[2]; k < b1[2]; ++k)
    for (int j = b0[1]; j < b1[1]; ++j)
      for (int i = b0[0]; i < b1[0]; ++i) {
        T f[27] = {};
        const int fi = (i - C.iS) * 2, fj = (j - C.jS) * 2, fk = (k - C.kS) * 2;
        for (int dk = 0; dk <= 1; ++dk)
          for (int dj = 0; dj <= 1; ++dj)
            for (int di = 0; di <= 1; ++di) {
              T g[27];
              readCell(gf, cellIndex(gf.info, fi + di, fj + dj, fk + dk), g);
              for (int q = 0; q < 27; ++q) f[q] += g[q];
            }
        for (int q = 0; q < 27; ++q) f[q] = f[q] * T(0.125);
        rescale(f, false);
        writeCell(gc, cellIndex(C, i, j, k), f);
      }
}

// gridRefinementFunctions.h:338-431: 7-point interpolation around the parent coarse cell
// (central differences, one-sided at the coarse domain edge), rescaled coarse->fine,
// written to fine cells of the box [b0, b1): all 27 populations, or only `dirs` (the 9
// that stream into the fine grid) on fine ghost cells.
template <typename T>
static void prolongBox(Sim<T>& sim, Grid<T>& gc, Grid<T>& gf, const int b0[3], const int b1[3], const int* dirs) {
  const Info& C = gc.info;
  const Info& F = gf.info;
  for (int k = b0[2]; k < b1[2]; ++k)
    for (int j = b0[1]; j < b1[1]; ++j)
      for (int i = b0[0]; i < b1[0]; ++i) {
        const int ic = i / 2 + C.iS, jc = j / 2 + C.jS, kc = k / 2 + C.kS;
        const T d[3] = {(i % 2) ? T(0.25) : T(-0.25), (j % 2) ? T(0.25) : T(-0.25), (k % 2) ? T(0.25) : T(-0.25)};
        T f[27];
        readCell(gc, cellIndex(C, ic, jc, kc), f);
        const int cc[3] = {ic, jc, kc};
        const int nmax[3] = {C.nx, C.ny, C.nz};
        for (int ax = 0; ax < 3; ++ax) {
          int plus = cc[ax] + 1, minus = cc[ax] - 1;
          T inv = T(0.5);
          if (plus >= nmax[ax]) { plus = cc[ax]; inv = T(1); }
          if (minus < 0) { minus = 0; inv = T(1); }
          int p[3] = {ic, jc, kc}, m[3] = {ic, jc, kc};
          p[ax] = plus;
          m[ax] = minus;
          T fp[27], fm[27];
          readCell(gc, cellIndex(C, p[0], p[1], p[2]), fp);
          readCell(gc, cellIndex(C, m[0], m[1], m[2]), fm);
          for (int q = 0; q < 27; ++q) f[q] += fp[q] * inv * d[ax];
          for (int q = 0; q < 27; ++q) f[q] += fm[q] * (-inv) * d[ax];
        }
        rescale(f, true);
        const long long cell = cellIndex(F, i, j, k);
        if (cellKind(sim.cfg, F, i, j, k) == Kind::Skip) {
          for (int r = 0; r < 9; ++r) gf.f[(size_t)dirs[r] * F.n + gf.addr(dirs[r], cell)] = f[dirs[r]];
        } else {
          writeCell(gf, cell, f);
        }
      }
}

// applyCoarseFineGridCommunication, gridRefinementFunctions.h:433-526.
template <typename T>
static void coarseFine(Sim<T>& sim, Grid<T>& gc, Grid<T>& gf) {
  const Info& C = gc.info;
  const Info& F = gf.info;
  static const int posX[9] = {1, 7, 9, 12, 16, 20, 22, 23, 26}, negX[9] = {2, 8, 10, 11, 15, 19, 21, 24, 25};
  static const int posY[9] = {6, 12, 13, 15, 17, 19, 22, 24, 26}, negY[9] = {5, 11, 14, 16, 18, 20, 21, 23, 25};
  static const int posZ[9] = {4, 8, 9, 14, 17, 20, 21, 24, 26}, negZ[9] = {3, 7, 10, 13, 18, 19, 22, 23, 25};
  const int lo[3] = {C.iS + 1, C.jS + 1, C.kS + 1};
  const int hi[3] = {C.iE - 1, C.jE - 1, C.kE - 1};
  const int ncoarse[3] = {C.nx, C.ny, C.nz};
  const int endIdx[3] = {C.iE - 2, C.jE - 2, C.kE - 2};
  for (int ax = 0; ax < 3; ++ax) {
    if (ncoarse[ax] <= 1) continue;
    int b0[3] = {lo[0], lo[1], lo[2]}, b1[3] = {hi[0], hi[1], hi[2]};
    b1[ax] = lo[ax] + 1;
    restrictBox(gc, gf, b0, b1);
    b0[ax] = endIdx[ax];
    b1[ax] = endIdx[ax] + 1;
    restrictBox(gc, gf, b0, b1);
  }
  const int startS[3] = {C.iS, C.jS, C.kS};
  const int endS[3] = {C.iE, C.jE, C.kE};
  const int nf[3] = {F.nx, F.ny, F.nz};
  const int* pos[3] = {posX, posY, posZ};
  const int* neg[3] = {negX, negY, negZ};
  for (int ax = 0; ax < 3; ++ax) {
    if (startS[ax] > 0) {
      int b0[3] = {0, 0, 0}, b1[3] = {nf[0], nf[1], nf[2]};
      b1[ax] = 2;
      prolongBox(sim, gc, gf, b0, b1, pos[ax]);
    }
    if (endS[ax] < ncoarse[ax] - 1) {
      int b0[3] = {0, 0, 0}, b1[3] = {nf[0], nf[1], nf[2]};
      b0[ax] = nf[ax] - 2;
      prolongBox(sim, gc, gf, b0, b1, neg[ax]);
    }
  }
}

template <typename T>
static void updateLevel(Sim<T>& sim, int level) {  // flowAroundSphereMainSingle.cu:158-167
  Grid<T>& g = sim.grids[level];
  streamShifts(g.shift, g.info);
  localUpdate(sim, g);
  if (level + 1 < (int)sim.grids.size()) {
    updateLevel(sim, level + 1);
    updateLevel(sim, level + 1);
    coarseFine(sim, g, sim.grids[level + 1]);
  }
}

// fillEquilibrium.h:1-22 with the noisy-inflow start hook; solid cells start at rest.
template <typename T>
static void fillEquilibrium(Sim<T>& sim, Grid<T>& g) {
  const Info& I = g.info;
  const CaseConfig& c = sim.cfg;
#pragma omp parallel for schedule(static)
  for (long long cell = 0; cell < I.n; ++cell) {
    const int i = (int)(cell % I.nx), j = (int)((cell / I.nx) % I.ny), k = (int)(cell / ((long long)I.nx * I.ny));
    const bool solid = cellKind(c, I, i, j, k) == Kind::Solid;
    const float ux = solid ? 0.f : psl_noisy_velocity(c.uIn, c.noiseAmp, c.seed, (uint32_t)I.level, (uint32_t)cell, 0);
    const float uy = solid ? 0.f : psl_noisy_velocity(0.f, c.noiseAmp, c.seed, (uint32_t)I.level, (uint32_t)cell, 1);
    const float uz = solid ? 0.f : psl_noisy_velocity(0.f, c.noiseAmp, c.seed, (uint32_t)I.level, (uint32_t)cell, 2);
    T fe[27];
    feq(T(1), T(ux), T(uy), T(uz), fe);
    for (int q = 0; q < 27; ++q) g.f[(size_t)q * I.n + cell] = fe[q];
  }
}

template <typename T>
static Sim<T>* create(const CaseConfig& cfg) {
  Sim<T>* sim = new Sim<T>();
  sim->cfg = cfg;
  sim->grids.resize(cfg.levels);
  Info& c = sim->grids[0].info;
  c.level = 0;
  c.nx = cfg.nx; c.ny = cfg.ny; c.nz = cfg.nz;
  c.n = (long long)cfg.nx * cfg.ny * cfg.nz;
  c.nu = cfg.nuCoarse;
  if (cfg.levels > 1) {
    c.iS = cfg.iSub0; c.jS = cfg.jSub0; c.kS = cfg.kSub0;
    c.iE = cfg.iSub1; c.jE = cfg.jSub1; c.kE = cfg.kSub1;
  }
  for (int l = 1; l < cfg.levels; ++l) {
    const Info& p = sim->grids[l - 1].info;
    Info& f = sim->grids[l].info;
    f.level = l;
    f.res = p.res * 0.5f;
    f.nu = p.nu * 2.f;
    f.ox = p.ox + p.iS * p.res - f.res * 0.5f;
    f.oy = p.oy + p.jS * p.res - f.res * 0.5f;
    f.oz = p.oz + p.kS * p.res - f.res * 0.5f;
    f.nx = (p.iE - p.iS) * 2; f.ny = (p.jE - p.jS) * 2; f.nz = (p.kE - p.kS) * 2;
    f.n = (long long)f.nx * f.ny * f.nz;
    if (l + 1 < cfg.levels) {  // the next finer block lies on this grid
      f.iS = cfg.iSub2_0; f.jS = cfg.jSub2_0; f.kS = cfg.kSub2_0;
      f.iE = cfg.iSub2_1; f.jE = cfg.jSub2_1; f.kE = cfg.kSub2_1;
    }
  }
  for (auto& g : sim->grids) {
    g.f.assign((size_t)27 * (size_t)g.info.n, T(0));
    fillEquilibrium(*sim, g);
  }
  return sim;
}

// Momentum-exchange drag on the finest grid (flowAroundSphereMainSingle.cu:99-156),
// per-cell contributions in T, accumulated in double.
template <typename T>
static double dragLattice(Sim<T>& sim) {
  Grid<T>& g = sim.grids.back();
  const Info& I = g.info;
  const CaseConfig& c = sim.cfg;
  const int i0 = (int)((c.sphereX - c.sphereR - I.ox) / I.res), i1 = (int)((c.sphereX + c.sphereR - I.ox) / I.res) + 2;
  const int j0 = (int)((c.sphereY - c.sphereR - I.oy) / I.res), j1 = (int)((c.sphereY + c.sphereR - I.oy) / I.res) + 2;
  const int k0 = (int)((c.sphereZ - c.sphereR - I.oz) / I.res), k1 = (int)((c.sphereZ + c.sphereR - I.oz) / I.res) + 2;
  double acc = 0.0;
  for (int k = k0; k < k1; ++k)
    for (int j = j0; j < j1; ++j)
      for (int i = i0; i < i1; ++i) {
        if (cellKind(c, I, i, j, k) != Kind::Solid) continue;
        T f[27];
        readCell(g, cellIndex(I, i, j, k), f);
        T rho, ux, uy, uz;
        rhoU(f, rho, ux, uy, uz);
        bounceback(f);
        T r2, ux2, uy2, uz2;
        rhoU(f, r2, ux2, uy2, uz2);
        acc += (double)(rho * (ux - ux2));
      }
  return acc;
}

}  // namespace oracle

// ------------------------------------------------------------------------------------------
// C API (ctypes)
// ------------------------------------------------------------------------------------------
using namespace oracle;

struct OracleHandle {
  int isDouble;
  Sim<float>* sf = nullptr;
  Sim<double>* sd = nullptr;
};

template <typename T>
static void getF(Grid<T>& g, T* out) {
  const long long N = g.info.n;
  for (int q = 0; q < 27; ++q)
    for (long long c = 0; c < N; ++c) out[(size_t)q * N + c] = g.f[(size_t)q * N + g.addr(q, c)];
}
template <typename T>
static void setF(Grid<T>& g, const T* in) {
  const long long N = g.info.n;
  for (int q = 0; q < 27; ++q)
    for (long long c = 0; c < N; ++c) g.f[(size_t)q * N + g.addr(q, c)] = in[(size_t)q * N + c];
}

extern "C" {

void* oracle_sim_create(const CaseConfig* cfg, int useDouble) {
  OracleHandle* h = new OracleHandle();
  h->isDouble = useDouble;
  if (useDouble) h->sd = create<double>(*cfg);
  else h->sf = create<float>(*cfg);
  return h;
}
void oracle_sim_destroy(void* p) {
  OracleHandle* h = static_cast<OracleHandle*>(p);
  delete h->sf;
  delete h->sd;
  delete h;
}
void oracle_sim_run(void* p, int steps) {
  OracleHandle* h = static_cast<OracleHandle*>(p);
  for (int s = 0; s < steps; ++s) {
    if (h->isDouble) updateLevel(*h->sd, 0);
    else updateLevel(*h->sf, 0);
  }
}
long long oracle_sim_cell_count(void* p, int level) {
  OracleHandle* h = static_cast<OracleHandle*>(p);
  return h->isDouble ? h->sd->grids[level].info.n : h->sf->grids[level].info.n;
}
void oracle_sim_get_f(void* p, int level, void* out) {
  OracleHandle* h = static_cast<OracleHandle*>(p);
  if (h->isDouble) getF(h->sd->grids[level], static_cast<double*>(out));
  else getF(h->sf->grids[level], static_cast<float*>(out));
}
void oracle_sim_set_f(void* p, int level, const void* in) {
  OracleHandle* h = static_cast<OracleHandle*>(p);
  if (h->isDouble) setF(h->sd->grids[level], static_cast<const double*>(in));
  else setF(h->sf->grids[level], static_cast<const float*>(in));
}
void oracle_sim_get_shifts(void* p, int level, int* out) {
  OracleHandle* h = static_cast<OracleHandle*>(p);
  for (int q = 0; q < 27; ++q)
    out[q] = (int)(h->isDouble ? h->sd->grids[level].shift[q] : h->sf->grids[level].shift[q]);
}
// fillCoarseGridFromFine (gridRefinementFunctions.h:528-535): restriction of the coarse box
// [iS+1, iE-1) x [jS+1, jE-1) x [kS+1, kE-1) of level `level` from level `level` + 1.
void oracle_sim_fill_coarse_from_fine(void* p, int level) {
  OracleHandle* h = static_cast<OracleHandle*>(p);
  auto fill = [level](auto& sim) {
    auto& gc = sim.grids[level];
    auto& gf = sim.grids[level + 1];
    const Info& C = gc.info;
    const int b0[3] = {C.iS + 1, C.jS + 1, C.kS + 1}, b1[3] = {C.iE - 1, C.jE - 1, C.kE - 1};
    restrictBox(gc, gf, b0, b1);
  };
  if (h->isDouble) fill(*h->sd);
  else fill(*h->sf);
}
double oracle_sim_drag(void* p) {
  OracleHandle* h = static_cast<OracleHandle*>(p);
  return h->isDouble ? dragLattice(*h->sd) : dragLattice(*h->sf);
}

// ---- single-function entry points, float and double ----
#define ORACLE_UNARY(T, SUF)                                                                            \
  void oracle_collision_##SUF(T* f, T nu, T cs) { collide<T>(f, nu, cs); }                             \
  void oracle_collision_forced_##SUF(T* f, T nu, T cs, T gx, T gy, T gz) { collide<T>(f, nu, cs, gx, gy, gz); } \
  void oracle_feq_##SUF(T rho, T ux, T uy, T uz, T* out) { feq<T>(rho, ux, uy, uz, out); }            \
  void oracle_rescale_##SUF(T* f, int c2f) { rescale<T>(f, c2f != 0); }                               \
  void oracle_mbbc_##SUF(int n, T rho, T ux, T uy, T uz, T* f) { mbbc<T>(n, f, rho, ux, uy, uz); }    \
  void oracle_restore_rho_##SUF(int n, T ux, T uy, T uz, const T* f, T* rho) { restoreRho<T>(n, f, *rho, ux, uy, uz); } \
  void oracle_restore_u_##SUF(int n, T rho, const T* f, T* u) { restoreU<T>(n, f, rho, u[0], u[1], u[2]); } \
  void oracle_restore_rho_u_##SUF(int n, const T* f, T* o) { restoreRhoU<T>(n, f, o[0], o[1], o[2], o[3]); } \
  void oracle_mirror_##SUF(int n, T* f) { mirror<T>(n, f); }                                          \
  void oracle_bounceback_##SUF(T* f) { bounceback<T>(f); }                                            \
  void oracle_moving_bounceback_##SUF(T* f, T ux, T uy, T uz) { movingBounceback<T>(f, ux, uy, uz); } \
  T oracle_omega_les_##SUF(const T* f, T nu, T cs) {                                                  \
    T rho, ux, uy, uz;                                                                                \
    rhoU<T>(f, rho, ux, uy, uz);                                                                      \
    return omegaLES<T>(f, rho, ux, uy, uz, nu, cs);                                                   \
  }

ORACLE_UNARY(float, f32)
ORACLE_UNARY(double, f64)

void oracle_streaming(int nx, int ny, int nz, int* shifts) {
  Info I;
  I.nx = nx; I.ny = ny; I.nz = nz;
  I.n = (long long)nx * ny * nz;
  long long s[27];
  for (int q = 0; q < 27; ++q) s[q] = shifts[q];
  streamShifts(s, I);
  for (int q = 0; q < 27; ++q) shifts[q] = (int)s[q];
}

}  // extern "C"
