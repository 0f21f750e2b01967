// C ABI of the learned subgrid closure (include/psl.h, psl_set_sgs_mlp / psl_sgs_mlp_infer)
// and the launch of the update kernel that fuses it (psl_learned.cuh).
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstring>
#include <string>

#include "psl.h"
#include "psl_internal.h"
#include "psl_learned.cuh"

using namespace psl;

namespace {

int fail(int code, const std::string& msg) {
  psl_detail_set_last_error(msg);
  return code;
}

#define MLP_CUDA(expr)                                                                                 \
  do {                                                                                                 \
    cudaError_t e_ = (expr);                                                                           \
    if (e_ != cudaSuccess) return fail(PSL_ERR_CUDA, std::string(#expr) + ": " + cudaGetErrorString(e_)); \
  } while (0)

// The grid's closure buffer: the tcgen05 layout followed by the per-warp layout.
struct MlpBoth {
  MlpDevice cta;
  MlpFrag warp;
};
static_assert(sizeof(MlpScalars) <= sizeof(float) * 24, "psl_grid::mlp_scalars holds MlpScalars");

// FP16 pair (lo, hi) as one 32-bit fragment register.
uint32_t half_pair(float lo, float hi) {
  const __half a = __float2half_rn(lo), b = __float2half_rn(hi);
  uint16_t ua, ub;
  std::memcpy(&ua, &a, 2);
  std::memcpy(&ub, &b, 2);
  return (uint32_t)ua | ((uint32_t)ub << 16);
}

// Per-warp layout: every lane's B fragments in the order mlp_warp_eval loads them
// (psl_mlp_warp.cuh); W(o, k) gives the weight of output o, input k.
template <typename Wfn>
uint4 frag_pair(Wfn W, int np, int kk, int lane) {
  const int g = lane >> 2, t = lane & 3;
  auto b0 = [&](int nt) { return half_pair(W(8 * nt + g, 16 * kk + 2 * t), W(8 * nt + g, 16 * kk + 2 * t + 1)); };
  auto b1 = [&](int nt) { return half_pair(W(8 * nt + g, 16 * kk + 8 + 2 * t), W(8 * nt + g, 16 * kk + 9 + 2 * t)); };
  return make_uint4(b0(2 * np), b1(2 * np), b0(2 * np + 1), b1(2 * np + 1));
}

void pack_warp(const psl_sgs_mlp& m, MlpFrag& d, MlpScalars& sc) {
  std::memset(&d, 0, sizeof(d));
  auto w1 = [&](int o, int k) { return k < kMlpIn ? m.w1[o][k] : (k == kMlpIn ? m.b1[o] : 0.f); };
  auto w2 = [&](int o, int k) { return m.w2[o][k]; };
  auto w3 = [&](int o, int k) { return o == 0 ? m.w3[k] : 0.f; };
  for (int lane = 0; lane < 32; ++lane) {
    const int t = lane & 3;
    for (int np = 0; np < 2; ++np) {
      d.w1[np][lane] = frag_pair(w1, np, 0, lane);
      for (int kk = 0; kk < 2; ++kk) d.w2[kk][np][lane] = frag_pair(w2, np, kk, lane);
    }
    const uint4 k0 = frag_pair(w3, 0, 0, lane), k1 = frag_pair(w3, 0, 1, lane);
    d.w3[lane] = make_uint4(k0.x, k0.y, k1.x, k1.y);  // N-tile 0 of K-steps 0 and 1
    for (int kk = 0; kk < 2; ++kk) {
      const int c = 16 * kk + 2 * t;
      d.b2[kk][lane] = make_float4(m.b2[c], m.b2[c + 1], m.b2[c + 8], m.b2[c + 9]);
    }
  }
  std::memset(&sc, 0, sizeof(sc));
  sc.b3 = m.b3;
  sc.out_scale = m.out_scale;
  for (int i = 0; i < kMlpIn; ++i) {
    sc.in_scale[i] = m.in_scale[i];
    sc.in_offset[i] = -m.in_shift[i] * m.in_scale[i];
  }
}

// FP16 weights in the tcgen05 operand layout, FP32 biases and normalisation.
void pack(const psl_sgs_mlp& m, MlpDevice& d) {
  std::memset(&d, 0, sizeof(d));
  auto put = [](__half* base, uint32_t rows, uint32_t r, uint32_t k, float v) {
    base[mlp_operand_offset(rows, r, k) / 2] = __float2half_rn(v);
  };
  for (int r = 0; r < kMlpHidden; ++r) {
    for (int k = 0; k < kMlpK1; ++k)
      put(d.w1, kMlpHidden, r, k, k < kMlpIn ? m.w1[r][k] : (k == kMlpIn ? m.b1[r] : 0.f));
    for (int k = 0; k < kMlpHidden; ++k) put(d.w2, kMlpHidden, r, k, m.w2[r][k]);
  }
  for (int r = 0; r < kMlpN3; ++r)
    for (int k = 0; k < kMlpHidden; ++k) put(d.w3, kMlpN3, r, k, r == 0 ? m.w3[k] : 0.f);
  for (int i = 0; i < kMlpHidden; ++i) d.b2[i] = m.b2[i];
  d.b3 = m.b3;
  d.out_scale = m.out_scale;
  for (int i = 0; i < kMlpIn; ++i) {
    d.in_scale[i] = m.in_scale[i];
    d.in_offset[i] = -m.in_shift[i] * m.in_scale[i];
  }
}

template <typename S>
int launch(psl_grid* g, const ThreadRange& range) {
  const MlpBoth* both = static_cast<const MlpBoth*>(g->mlp);
  MlpScalars sc;
  std::memcpy(&sc, g->mlp_scalars, sizeof(MlpScalars));
  if (27ull * g->f_stride + g->n >= (1ull << 32)) return fail(PSL_ERR_INVALID, "learned update: grid too large");
  LearnedParams<S> p;
  p.ri.base = static_cast<typename S::type*>(g->f);
  p.ri.n = g->n;
  for (int q = 0; q < 27; ++q) {
    p.ri.off[q] = (uint32_t)((size_t)q * g->f_stride + g->shift[q]);
    p.ri.lim[q] = g->n - g->shift[q];
  }
  p.marker = g->marker;
  p.given = g->given;
  p.given_uniform = g->given_uniform;
  p.mlpw = &both->warp;
  p.sc = sc;
  p.nu = g->info.nu;
  p.width = g->mlp_width;
  p.n = g->n;
  p.health = g->health;
  p.rot = psl_detail_thread_rotation(g);
  p.nut = g->mlp_nut;
  p.range = range;
  const unsigned int blocks = (range.count + kStepThreads - 1) / kStepThreads;
  auto go = [&](auto kernel) { kernel<<<blocks, kStepThreads, 0, g->stream>>>(p); };
  if constexpr (kCollidesOnG<S>) {
    if (g->mlp_nut) {  // evaluated every mlp_interval-th update: keep nu_t for the others
      g->f_twice ? go(step_learned_warp_kernel<S, true, true>) : go(step_learned_warp_kernel<S, false, true>);
      MLP_CUDA(cudaGetLastError());
      return PSL_OK;
    }
  }
  g->f_twice ? go(step_learned_warp_kernel<S, true, false>) : go(step_learned_warp_kernel<S, false, false>);
  MLP_CUDA(cudaGetLastError());
  return PSL_OK;
}

}  // namespace

int psl_detail_launch_learned(psl_grid* g, const ThreadRange& range) {
  switch (g->storage) {
    case kStoreF32: return launch<StoreF32>(g, range);
    case kStoreF16: return launch<StoreF16>(g, range);
    case kStoreBF16: return launch<StoreBF16>(g, range);
    default: return fail(PSL_ERR_INVALID, "learned update: FP64 storage is for oracle runs only");
  }
}

int psl_set_sgs_mlp(psl_grid* g, const psl_sgs_mlp* mlp, float filter_width) {
  if (!g) return fail(PSL_ERR_INVALID, "psl_set_sgs_mlp: null grid");
  DeviceGuard dg(g->device);
  psl_detail_closure_stale(g);
  if (!mlp) {
    if (g->mlp) {
      MLP_CUDA(cudaStreamSynchronize(g->stream));
      cudaFree(g->mlp);
      g->mlp = nullptr;
    }
    return PSL_OK;
  }
  if (g->storage == kStoreF64) return fail(PSL_ERR_INVALID, "psl_set_sgs_mlp: FP64 storage is for oracle runs only");
  MlpBoth host;
  MlpScalars sc;
  pack(*mlp, host.cta);
  pack_warp(*mlp, host.warp, sc);
  if (!g->mlp) {
    cudaError_t e = cudaMalloc(&g->mlp, sizeof(MlpBoth));
    if (e != cudaSuccess) {
      g->mlp = nullptr;
      cudaGetLastError();
      return fail(PSL_ERR_NOMEM, std::string("psl_set_sgs_mlp: ") + cudaGetErrorString(e));
    }
  }
  MLP_CUDA(cudaMemcpyAsync(g->mlp, &host, sizeof(MlpBoth), cudaMemcpyHostToDevice, g->stream));
  MLP_CUDA(cudaStreamSynchronize(g->stream));
  g->mlp_width = filter_width;
  std::memcpy(g->mlp_scalars, &sc, sizeof(MlpScalars));
  return PSL_OK;
}

int psl_set_sgs_mlp_interval(psl_grid* g, int interval) {
  if (!g) return fail(PSL_ERR_INVALID, "psl_set_sgs_mlp_interval: null grid");
  if (interval < 1) return fail(PSL_ERR_INVALID, "psl_set_sgs_mlp_interval: the interval must be at least 1");
  if (interval > 1 && g->storage != kStoreF16 && g->storage != kStoreBF16)
    return fail(PSL_ERR_INVALID, "psl_set_sgs_mlp_interval: intervals above 1 need FP16 or BF16 storage");
  DeviceGuard dg(g->device);
  if (interval == 1) {
    if (g->mlp_nut) {
      MLP_CUDA(cudaStreamSynchronize(g->stream));
      cudaFree(g->mlp_nut);
      g->mlp_nut = nullptr;
    }
  } else if (!g->mlp_nut) {
    cudaError_t e = cudaMalloc(&g->mlp_nut, (size_t)g->n * sizeof(uint16_t));
    if (e != cudaSuccess) {
      g->mlp_nut = nullptr;
      cudaGetLastError();
      return fail(PSL_ERR_NOMEM, std::string("psl_set_sgs_mlp_interval: ") + cudaGetErrorString(e));
    }
  }
  g->mlp_interval = interval;
  psl_detail_closure_stale(g);
  return PSL_OK;
}

int psl_sgs_mlp_infer(const psl_sgs_mlp* mlp, const float* features, int count, float* nu_t) {
  if (!mlp || !features || !nu_t || count <= 0) return fail(PSL_ERR_INVALID, "psl_sgs_mlp_infer: bad argument");
  int ndev = 0;
  MLP_CUDA(cudaGetDeviceCount(&ndev));
  if (ndev <= 0) return fail(PSL_ERR_CUDA, "psl_sgs_mlp_infer: no CUDA device");
  MlpDevice host;
  pack(*mlp, host);
  MlpDevice* dm = nullptr;
  float *dx = nullptr, *dy = nullptr;
  unsigned int* dh = nullptr;
  cudaError_t e = cudaMalloc(&dm, sizeof(MlpDevice));
  if (e == cudaSuccess) e = cudaMalloc(&dx, (size_t)count * kMlpIn * sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc(&dy, (size_t)count * sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc(&dh, sizeof(unsigned int));
  if (e == cudaSuccess) e = cudaMemset(dh, 0, sizeof(unsigned int));
  if (e == cudaSuccess) e = cudaMemcpy(dm, &host, sizeof(MlpDevice), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(dx, features, (size_t)count * kMlpIn * sizeof(float), cudaMemcpyHostToDevice);
  unsigned int health = 0;
  if (e == cudaSuccess) {
    mlp_infer_kernel<<<(count + kMlpRows - 1) / kMlpRows, kMlpRows>>>(dm, dx, count, dy, dh);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpy(nu_t, dy, (size_t)count * sizeof(float), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(&health, dh, sizeof(unsigned int), cudaMemcpyDeviceToHost);
  cudaFree(dm);
  cudaFree(dx);
  cudaFree(dy);
  cudaFree(dh);
  if (e != cudaSuccess) return fail(PSL_ERR_CUDA, std::string("psl_sgs_mlp_infer: ") + cudaGetErrorString(e));
  if (health) return fail(PSL_ERR_STATE, "psl_sgs_mlp_infer: a tensor-core wait timed out");
  return PSL_OK;
}
