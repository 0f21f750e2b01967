// Per-case hooks, in the reference's shape.
//
// A reference case defines free functions getMarkers, getGivenRhoUxUyUz,
// getSmagorinskyConstant and getInitialRhoUxUyUz before including the solver headers
// (flowAroundSphere/flowAroundSphereMainSingle.cu:41-92).  Here a case is a small struct
// with the same four member functions (same arguments and meaning), passed by value to
// templated set-up kernels:
//
//   fill_markers_kernel<Case>    evaluates getMarkers / getGivenRhoUxUyUz once per cell and
//                                stores a one-byte marker (+ optional given values);
//   fill_equilibrium_kernel<Case> evaluates getInitialRhoUxUyUz (fillEquilibrium.h:1-22).
//
// The per-step kernel then reads the marker byte instead of re-evaluating the hooks for
// every cell on every step.  A case whose hooks change over time re-runs the set-up
// kernels when they change.
#pragma once
#include <stdint.h>

#include "psl_case_noise.h"
#include "psl_lattice.cuh"

namespace psl {

// Mirrors InfoStruct (include/types.h:73-75): the per-grid metadata hooks receive.
struct InfoStruct {
  float gridID = 0;
  float res = 1.f;
  int cellCountX = 0, cellCountY = 0, cellCountZ = 0;
  int cellCount = 0;
  float ox = 0.f, oy = 0.f, oz = 0.f;
  float nu = 1.f;
  float dtPhys = 1.f;
  int iSubgridStart = 0, jSubgridStart = 0, kSubgridStart = 0;
  int iSubgridEnd = 0, jSubgridEnd = 0, kSubgridEnd = 0;
};

// Mirrors MarkerStruct (include/types.h:79-80) plus the free-slip flag that the
// reference's free-slip wiring reads (include/scalarTransportFunctions.h:74).
struct MarkerStruct {
  bool fluid = 0, bounceback = 0, movingBounceback = 0, forcedVelocity = 0;
  bool periodicX = 0, periodicY = 0, periodicZ = 0;
  bool givenRho = 0, givenUxUyUz = 0, nonReflectiveOutlet = 0, refinement = 0, ghost = 0;
  bool mirror = 0;
};

// getOuterNormal (include/cellFunctions.h:46-58)
PSL_HDI void getOuterNormal(int i, int j, int k, int& nx, int& ny, int& nz, const InfoStruct& I) {
  nx = (i == 0) ? -1 : (i == I.cellCountX - 1 ? 1 : 0);
  ny = (j == 0) ? -1 : (j == I.cellCountY - 1 ? 1 : 0);
  nz = (k == 0) ? -1 : (k == I.cellCountZ - 1 ? 1 : 0);
}

// Encode the marker byte exactly as applyLocalCellUpdate.h:21-67 interprets the hooks:
// ghost and refined-interior cells are skipped first, then bounce-back, fluid, and the
// boundary kinds with the outer normal (periodic components zeroed).  A skipped cell keeps
// the hook's bounce-back flag in its normal bits (kSkipSolid) for the exports, which report
// getMarkers' bounceback on every cell (plotter/exportSectionCutPlot.h:45-48).
PSL_HDI uint8_t encode_marker(int i, int j, int k, const MarkerStruct& M, const InfoStruct& I) {
  if (M.ghost) return make_marker(kSkip, 1);
  if ((i > I.iSubgridStart + 1 && i < I.iSubgridEnd - 2) && (j > I.jSubgridStart + 1 && j < I.jSubgridEnd - 2) &&
      (k > I.kSubgridStart + 1 && k < I.kSubgridEnd - 2))
    return make_marker(kSkip, M.bounceback ? kSkipSolid : 0);
  if (M.movingBounceback) return make_marker(kSolid, 1);  // moving wall (customised update)
  if (M.bounceback) return make_marker(kSolid, 0);
  if (M.fluid) return make_marker(kFluid, M.forcedVelocity ? 1 : 0);  // 1: forced velocity
  int nx, ny, nz;
  getOuterNormal(i, j, k, nx, ny, nz, I);
  if (M.periodicX) nx = 0;
  if (M.periodicY) ny = 0;
  if (M.periodicZ) nz = 0;
  const int n = normal_index(nx, ny, nz);
  if (M.mirror) return make_marker(kMirror, n);
  if (M.givenRho && !M.givenUxUyUz) return make_marker(kGivenRho, n);
  if (!M.givenRho && M.givenUxUyUz) return make_marker(kGivenU, n);
  if (!M.givenRho && !M.givenUxUyUz) return make_marker(kGivenNone, n);
  return make_marker(kGivenBoth, n);
}

// ---- the flow-past-sphere case (flowAroundSphere/flowAroundSphereMainSingle.cu:41-92) ----
struct SphereCase {
  float sx, sy, sz, r;   // sphere centre and radius, physical units
  float uIn;             // inlet velocity (lattice units; also the given velocity)
  float rhoGiven;        // given density (outlet)
  int wallMode;          // 0: free-slip y/z walls, inlet/outlet planes first; 1: velocity walls
  float smagorinsky;
  uint32_t seed;
  float noiseAmp;

  __device__ void getMarkers(int i, int j, int k, MarkerStruct& M, const InfoStruct& I) const {
    const float x = i * I.res + I.ox, y = j * I.res + I.oy, z = k * I.res + I.oz;
    const float r2 = (x - sx) * (x - sx) + (y - sy) * (y - sy) + (z - sz) * (z - sz);
    if (I.gridID != 0) {
      if (r2 <= r * r) M.bounceback = 1;
      else if (i == 0 || i == I.cellCountX - 1) M.ghost = 1;
      else if (j == 0 || j == I.cellCountY - 1) M.ghost = 1;
      else if (k == 0 || k == I.cellCountZ - 1) M.ghost = 1;
      else M.fluid = 1;
      return;
    }
    if (r2 <= r * r) { M.bounceback = 1; return; }
    const bool wall = (j == 0 || j == I.cellCountY - 1 || k == 0 || k == I.cellCountZ - 1);
    if (wallMode == 1) {
      if (wall || i == 0) M.givenUxUyUz = 1;
      else if (i == I.cellCountX - 1) M.givenRho = 1;
      else M.fluid = 1;
    } else {
      if (i == 0) M.givenUxUyUz = 1;
      else if (i == I.cellCountX - 1) M.givenRho = 1;
      else if (wall) M.mirror = 1;
      else M.fluid = 1;
    }
  }
  __device__ void getGivenRhoUxUyUz(int, int, int, float& rho, float& ux, float& uy, float& uz,
                                    const InfoStruct&) const {
    rho = rhoGiven;
    ux = uIn;
    uy = 0.f;
    uz = 0.f;
  }
  __device__ float getSmagorinskyConstant(int, int, int, const InfoStruct&) const { return smagorinsky; }
  // feq(1, u_in + seeded noise): the noisy-inflow start of the sphere configurations.
  // Solid cells start at rest (the variant the reference driver keeps commented out at
  // flowAroundSphereMainSingle.cu:86-87), so the bounce-back interior of the sphere
  // carries no momentum into the momentum-exchange drag sum.
  __device__ void getInitialRhoUxUyUz(int i, int j, int k, float& rho, float& ux, float& uy, float& uz,
                                      const MarkerStruct& M, const InfoStruct& I) const {
    const uint32_t cell = (uint32_t)(((long long)k * I.cellCountY + j) * I.cellCountX + i);
    const uint32_t level = (uint32_t)I.gridID;
    rho = 1.f;
    if (M.bounceback) {
      ux = uy = uz = 0.f;
      return;
    }
    ux = psl_noisy_velocity(uIn, noiseAmp, seed, level, cell, 0);
    uy = psl_noisy_velocity(0.f, noiseAmp, seed, level, cell, 1);
    uz = psl_noisy_velocity(0.f, noiseAmp, seed, level, cell, 2);
  }
};

// ---- a uniform start state (fillEquilibrium with a constant hook) ----
struct UniformCase {
  float rho0, ux0, uy0, uz0;
  __device__ void getMarkers(int, int, int, MarkerStruct& M, const InfoStruct&) const { M.fluid = 1; }
  __device__ void getInitialRhoUxUyUz(int, int, int, float& rho, float& ux, float& uy, float& uz, const MarkerStruct&,
                                      const InfoStruct&) const {
    rho = rho0;
    ux = ux0;
    uy = uy0;
    uz = uz0;
  }
};

}  // namespace psl
