// D3Q27 lattice constants and the per-cell marker encoding shared by all kernels.
#pragma once
#include <stdint.h>

#ifndef PSL_HDI
#if defined(__CUDACC__)
#define PSL_HDI __host__ __device__ __forceinline__
#else
#define PSL_HDI inline
#endif
#endif

namespace psl {

// Velocity ordering of the reference (include/applyStreaming.h:1-8): 0 rest, 1-6 faces,
// 7-18 edges, 19-26 corners; opposite pairs are (1,2), (3,4), ..., (25,26).
//   cx: { 0, 1,-1, 0, 0, 0, 0, 1,-1, 1,-1,-1, 1, 0, 0,-1, 1, 0, 0,-1, 1,-1, 1, 1,-1,-1, 1 }
//   cy: { 0, 0, 0, 0, 0,-1, 1, 0, 0, 0, 0,-1, 1, 1,-1, 1,-1, 1,-1, 1,-1,-1, 1,-1, 1,-1, 1 }
//   cz: { 0, 0, 0,-1, 1, 0, 0,-1, 1, 1,-1, 0, 0,-1, 1, 0, 0, 1,-1,-1, 1, 1,-1,-1, 1,-1, 1 }
// Each component is stored as 2-bit fields (c + 1) of one 64-bit constant, so cx(q) with a
// compile-time q folds to an immediate in device code (no constant-memory table).
constexpr unsigned long long kPackCx = 0x20a21616089549ull;
constexpr unsigned long long kPackCy = 0x2220888a156155ull;
constexpr unsigned long long kPackCz = 0x220a09614a1615ull;
PSL_HDI constexpr int cx(int q) { return (int)((kPackCx >> (2 * q)) & 3ull) - 1; }
PSL_HDI constexpr int cy(int q) { return (int)((kPackCy >> (2 * q)) & 3ull) - 1; }
PSL_HDI constexpr int cz(int q) { return (int)((kPackCz >> (2 * q)) & 3ull) - 1; }

// Lattice weights w_q (include/cellFunctions.h:16).
PSL_HDI constexpr float lattice_weight(int q) {
  return q == 0 ? 8.f / 27.f : (q <= 6 ? 2.f / 27.f : (q <= 18 ? 1.f / 54.f : 1.f / 216.f));
}

// The same weights in the arithmetic type T (the FP64 form rounds 8/27 etc. in double).
template <typename T>
PSL_HDI constexpr T weight_t(int q) {
  return q == 0 ? T(8) / T(27) : (q <= 6 ? T(2) / T(27) : (q <= 18 ? T(1) / T(54) : T(1) / T(216)));
}

PSL_HDI constexpr int opposite(int q) { return q == 0 ? 0 : ((q & 1) ? q + 1 : q - 1); }

// Population index of velocity (x, y, z) in {-1,0,1}^3 ("slot" of the central-moment
// transform): 5-bit fields, one 64-bit constant per x slot, field 3*(y+1) + (z+1).
constexpr unsigned long long kPackSlot0 = 0x187cd0255579ull;
constexpr unsigned long long kPackSlot1 = 0x11334801b8b2ull;
constexpr unsigned long long kPackSlot2 = 0x1a659213d217ull;
PSL_HDI constexpr int slot(int i, int j, int k) {
  return (int)(((i == 0 ? kPackSlot0 : (i == 1 ? kPackSlot1 : kPackSlot2)) >> (5 * (3 * j + k))) & 31ull);
}

// Bit mask of the directions whose `axis` component equals `sign`.
PSL_HDI constexpr uint32_t dir_mask(int axis, int sign) {
  uint32_t m = 0;
  for (int q = 0; q < 27; ++q) {
    const int c = axis == 0 ? cx(q) : (axis == 1 ? cy(q) : cz(q));
    if (c == sign) m |= 1u << q;
  }
  return m;
}

// Per-cell marker byte: low 3 bits kind, high 5 bits outer-normal index
// ((nx+1)*9 + (ny+1)*3 + (nz+1), with the components of periodic directions zeroed).
enum CellKind : uint8_t {
  kSkip = 0,       // ghost or refined-interior cell: not updated (applyLocalCellUpdate.h:25-30)
  kFluid = 1,
  kSolid = 2,      // full-way bounce-back, no collision
  kGivenU = 3,     // velocity given: restoreRho + moment-based BC
  kGivenRho = 4,   // density given: restoreUxUyUz + moment-based BC
  kGivenNone = 5,  // neither given: restoreRhoUxUyUz + moment-based BC
  kGivenBoth = 6,  // both given: moment-based BC only
  kMirror = 7,     // free-slip wall: specular reflection of the unknown populations
};

PSL_HDI uint8_t make_marker(int kind, int normal) { return (uint8_t)((kind & 7) | (normal << 3)); }

// Normal bits of skipped cells: 1 ghost layer, kSkipSolid a refined-interior cell that the
// case marks bounce-back (not updated; solid for the exports), 0 other refined-interior cells.
constexpr int kSkipSolid = 2;
PSL_HDI int marker_kind(uint8_t m) { return m & 7; }
PSL_HDI int marker_normal(uint8_t m) { return m >> 3; }
// Whether the case marks the cell bounce-back (the exports' solid flag), updated or not.
PSL_HDI bool marker_solid(uint8_t m) {
  return marker_kind(m) == kSolid || (marker_kind(m) == kSkip && marker_normal(m) == kSkipSolid);
}
PSL_HDI constexpr int normal_index(int nx, int ny, int nz) { return (nx + 1) * 9 + (ny + 1) * 3 + (nz + 1); }

}  // namespace psl
