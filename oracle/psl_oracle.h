// CPU oracle: the project's own restatement of PeriodicShiftLBM's per-step lattice update.
//
// ORACLE / TEST INFRASTRUCTURE ONLY -- the checker, never the thing measured or shipped.
// Templated on the arithmetic type: T = float reproduces the reference's FP32 update (and
// is pinned against the reference's own code compiled through oracle/tnl_shim, see
// oracle/ref_cases.cpp); T = double is the FP64 oracle for the reduced-precision storage
// forms.  Each function names the reference file:line it restates.
#pragma once
#include <cstdint>
#include <vector>

namespace oracle {

// D3Q27 ordering of the reference (include/applyStreaming.h:1-8,
// include/cellFunctions.h:3-16): 0 rest, 1-6 faces, 7-18 edges, 19-26 corners,
// opposite pairs (1,2), (3,4), ..., (25,26).
constexpr int CX[27] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, -1, 1, 0, 0, -1, 1, 0, 0, -1, 1, -1, 1, 1, -1, -1, 1};
constexpr int CY[27] = {0, 0, 0, 0, 0, -1, 1, 0, 0, 0, 0, -1, 1, 1, -1, 1, -1, 1, -1, 1, -1, -1, 1, -1, 1, -1, 1};
constexpr int CZ[27] = {0, 0, 0, -1, 1, 0, 0, -1, 1, 1, -1, 0, 0, -1, 1, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1, -1, 1};

template <typename T>
struct Weights {
  static T w(int q) {
    if (q == 0) return T(8) / T(27);
    if (q <= 6) return T(2) / T(27);
    if (q <= 18) return T(1) / T(54);
    return T(1) / T(216);
  }
};

// Case description shared with oracle/ref_cases.cpp (RefCaseConfig): flow past a sphere.
struct CaseConfig {
  int nx, ny, nz;
  int levels;
  int iSub0, jSub0, kSub0;
  int iSub1, jSub1, kSub1;
  float sphereX, sphereY, sphereZ, sphereR;
  float uIn;
  float nuCoarse;
  float smagorinsky;
  int wallMode;  // 0 free-slip (mirror) y/z walls, 1 velocity walls
  uint32_t seed;
  float noiseAmp;
  int iSub2_0, jSub2_0, kSub2_0;  // third level: refinement block on the level-1 grid
  int iSub2_1, jSub2_1, kSub2_1;
  int csMode;  // 0 uniform Smagorinsky constant, 1 outlet sponge on the coarse grid
  float forceR0, forceR1, forceOmega;  // forced-velocity annulus (read by the reference build's getTorque only)
};

// getSmagorinskyConstant of the sphere cases (oracle/ref_cases.cpp): csMode 1 raises C_s
// linearly from i = 3 Nx / 4 to four times its value at the outlet plane (coarse grid).
inline float smagorinskyConstant(const CaseConfig& c, int gridID, int nx, int i) {
  if (c.csMode == 1 && gridID == 0) {
    const int i0 = (3 * nx) / 4;
    if (i > i0) return c.smagorinsky * (1.f + 3.f * (float)(i - i0) / (float)(nx - 1 - i0));
  }
  return c.smagorinsky;
}

}  // namespace oracle
