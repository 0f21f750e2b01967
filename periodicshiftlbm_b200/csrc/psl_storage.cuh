// Population storage formats.  `type` is the element in HBM, `calc` the arithmetic type
// of the update (FP32 for every production form; FP64 only for the FP64 oracle runs).
//
//   F32            f_q stored as is                       (216 B moved per cell update)
//   F16 / BF16     f_q - w_q stored in 16 bits            (108 B per cell update)
//   F64            f_q stored as is, FP64 arithmetic      (432 B; oracle runs only)
//
// Storing the deviation from the lattice weight keeps the stored values small (|f - w|
// is O(u) relative to w), so the 16-bit formats spend their mantissa on the part that
// changes.
#pragma once
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "psl_lattice.cuh"

namespace psl {

enum StorageKind : int { kStoreF32 = 0, kStoreF16 = 1, kStoreBF16 = 2, kStoreF64 = 3 };

// Read-only loads of the update kernels with a 256-byte L2 prefetch hint: a warp reads 64
// (16-bit) or 128 (FP32) contiguous bytes of a row, and the warps of the next cells read
// the rest of the same lines.
__device__ __forceinline__ float ldg_row(const float* p) {
  float v;
  asm("ld.global.nc.L2::256B.f32 %0, [%1];" : "=f"(v) : "l"(p));
  return v;
}
__device__ __forceinline__ uint16_t ldg_row(const uint16_t* p) {
  uint16_t v;
  asm("ld.global.nc.L2::256B.b16 %0, [%1];" : "=h"(v) : "l"(p));
  return v;
}

struct StoreF32 {
  using type = float;
  using calc = float;
  static constexpr int kind = kStoreF32;
  template <int Q>
  __device__ __forceinline__ static float load(const float* p) { return *p; }
  template <int Q>
  __device__ __forceinline__ static void store(float* p, float v) { *p = v; }
  __device__ __forceinline__ static float load_q(const float* p, int) { return *p; }
  __device__ __forceinline__ static void store_q(float* p, float v, int) { *p = v; }
  // Update-kernel forms: each element is read once by its owning cell (read-only path)
  // and then overwritten by it (evict-first store).
  template <int Q>
  __device__ __forceinline__ static float load_once(const float* p) { return ldg_row(p); }
  template <int Q>
  __device__ __forceinline__ static void store_once(float* p, float v) { __stcs(p, v); }
};

struct StoreF16 {
  using type = __half;
  using calc = float;
  static constexpr int kind = kStoreF16;
  template <int Q>
  __device__ __forceinline__ static float load(const __half* p) { return __half2float(*p) + lattice_weight(Q); }
  template <int Q>
  __device__ __forceinline__ static void store(__half* p, float v) { *p = __float2half_rn(v - lattice_weight(Q)); }
  __device__ __forceinline__ static float load_q(const __half* p, int q) { return __half2float(*p) + lattice_weight(q); }
  __device__ __forceinline__ static void store_q(__half* p, float v, int q) { *p = __float2half_rn(v - lattice_weight(q)); }
  template <int Q>
  __device__ __forceinline__ static float load_once(const __half* p) { return __half2float(__ldg(p)) + lattice_weight(Q); }
  template <int Q>
  __device__ __forceinline__ static void store_once(__half* p, float v) {
    __stcs(reinterpret_cast<unsigned short*>(p), __half_as_ushort(__float2half_rn(v - lattice_weight(Q))));
  }
};

struct StoreBF16 {
  using type = __nv_bfloat16;
  using calc = float;
  static constexpr int kind = kStoreBF16;
  template <int Q>
  __device__ __forceinline__ static float load(const __nv_bfloat16* p) { return __bfloat162float(*p) + lattice_weight(Q); }
  template <int Q>
  __device__ __forceinline__ static void store(__nv_bfloat16* p, float v) { *p = __float2bfloat16_rn(v - lattice_weight(Q)); }
  __device__ __forceinline__ static float load_q(const __nv_bfloat16* p, int q) {
    return __bfloat162float(*p) + lattice_weight(q);
  }
  __device__ __forceinline__ static void store_q(__nv_bfloat16* p, float v, int q) {
    *p = __float2bfloat16_rn(v - lattice_weight(q));
  }
  template <int Q>
  __device__ __forceinline__ static float load_once(const __nv_bfloat16* p) {
    return __bfloat162float(__ldg(p)) + lattice_weight(Q);
  }
  template <int Q>
  __device__ __forceinline__ static void store_once(__nv_bfloat16* p, float v) {
    __stcs(reinterpret_cast<unsigned short*>(p), __bfloat16_as_ushort(__float2bfloat16_rn(v - lattice_weight(Q))));
  }
};

struct StoreF64 {
  using type = double;
  using calc = double;
  static constexpr int kind = kStoreF64;
  template <int Q>
  __device__ __forceinline__ static double load(const double* p) { return *p; }
  template <int Q>
  __device__ __forceinline__ static void store(double* p, double v) { *p = v; }
  __device__ __forceinline__ static double load_q(const double* p, int) { return *p; }
  __device__ __forceinline__ static void store_q(double* p, double v, int) { *p = v; }
  template <int Q>
  __device__ __forceinline__ static double load_once(const double* p) { return __ldg(p); }
  template <int Q>
  __device__ __forceinline__ static void store_once(double* p, double v) { __stcs(p, v); }
};

// The stored value itself as the cell's working value: f for FP32 / FP64, g = f - w for
// the 16-bit forms (which collide on g, psl_collision_g.cuh).
template <typename S>
struct StoredOf {
  using type = typename S::type;
  using calc = typename S::calc;
  template <int Q>
  __device__ __forceinline__ static calc load_once(const type* p) {
    if constexpr (S::kind == kStoreF16) return __half2float(__ldg(p));
    else if constexpr (S::kind == kStoreBF16) return __bfloat162float(__ldg(p));
    else return S::template load_once<Q>(p);
  }
  template <int Q>
  __device__ __forceinline__ static void store_once(type* p, calc v) {
    if constexpr (S::kind == kStoreF16) __stcs(reinterpret_cast<unsigned short*>(p), __half_as_ushort(__float2half_rn(v)));
    else if constexpr (S::kind == kStoreBF16)
      __stcs(reinterpret_cast<unsigned short*>(p), __bfloat16_as_ushort(__float2bfloat16_rn(v)));
    else S::template store_once<Q>(p, v);
  }
  template <int Q>
  __device__ __forceinline__ static calc load(const type* p) {
    if constexpr (S::kind == kStoreF16) return __half2float(*p);
    else if constexpr (S::kind == kStoreBF16) return __bfloat162float(*p);
    else return *p;
  }
  template <int Q>
  __device__ __forceinline__ static void store(type* p, calc v) {
    if constexpr (S::kind == kStoreF16) *p = __float2half_rn(v);
    else if constexpr (S::kind == kStoreBF16) *p = __float2bfloat16_rn(v);
    else *p = v;
  }
};

// Whether a storage form collides on the stored deviations g = f - w.
template <typename S>
constexpr bool kCollidesOnG = S::kind == kStoreF16 || S::kind == kStoreBF16;

// The 16 stored bits of a 16-bit form, unconverted: the update's fluid cells feed them to
// the moment sums directly (raw_moments_g_bits), solid cells swap them.
template <typename S>
struct StoredBits {
  static_assert(kCollidesOnG<S>, "16-bit storage forms only");
  using type = typename S::type;
  using calc = uint16_t;
  template <int Q>
  __device__ __forceinline__ static uint16_t load_once(const type* p) {
    return ldg_row(reinterpret_cast<const uint16_t*>(p));
  }
  template <int Q>
  __device__ __forceinline__ static void store_once(type* p, uint16_t v) {
    __stcs(reinterpret_cast<unsigned short*>(p), v);
  }
  template <int Q>
  __device__ __forceinline__ static uint16_t load(const type* p) { return *reinterpret_cast<const unsigned short*>(p); }
  template <int Q>
  __device__ __forceinline__ static void store(type* p, uint16_t v) { *reinterpret_cast<unsigned short*>(p) = v; }
  __device__ __forceinline__ static float to_float(uint16_t v) {
    if constexpr (S::kind == kStoreF16) return __half2float(__ushort_as_half(v));
    else return __bfloat162float(__ushort_as_bfloat16(v));
  }
};

inline size_t storage_bytes(int kind) { return kind == kStoreF32 ? 4 : kind == kStoreF64 ? 8 : 2; }

}  // namespace psl
