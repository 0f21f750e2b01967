// Training of the learned subgrid closure on the GPU (include/psl.h, psl_sgs_trainer_*):
// training samples filtered from fine-grid runs of this solver, the closure's forward and
// backward passes, a deterministic cross-block gradient reduction and Adam.
//
// Samples.  A fine periodic box of 2M physical cells per axis (grid 2M+1 x 2M+1 x 2M: the
// x and y faces are the duplicated layers of applyBCPeriodicX/Y, periodicXY.h:11-101; z
// wraps through the periodic shift) is box-filtered 2x to M^3 coarse cells:
//   * the 8 children's populations are averaged and rescaled fine -> coarse
//     (gridRefinementFunctions.h:6-281, the transfer the solver's own restriction uses);
//     the features are those the coarse solver's update kernel would compute from them;
//   * the target is the least-squares eddy viscosity of the filtered field,
//       nu_t* = max(0, -tau^d : S / (2 S : S)),
//     tau_ij = <u_i u_j> - <u>_i <u>_j over the 8 children, S the strain rate of the
//     filtered velocity (central differences, periodic), in coarse lattice units.
//
// Gradients.  The loss is the mean over a batch of (softplus(z) - nu_t*/out_scale)^2.  A
// block takes 128 samples at a time, one per thread: forward and backward per thread,
// then the block forms its weight gradients as sums over the 128 samples held in shared
// memory; blocks write partial gradients that one kernel sums in block order in FP64.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "psl.h"
#include "psl_internal.h"
#include "psl_kernels.cuh"
#include "psl_mlp.cuh"

using namespace psl;

namespace {

// flat parameter vector: w1 [32][10], b1 [32], w2 [32][32], b2 [32], w3 [32], b3, then the
// normalisation (in_shift [10], in_scale [10], out_scale), which training does not change
constexpr int kW1 = 0, kB1 = 320, kW2 = 352, kB2 = 1376, kW3 = 1408, kB3 = 1440, kTrainable = 1441;
constexpr int kShift = 1441, kScale = 1451, kOutScale = 1461, kParams = 1462;
constexpr int kGradThreads = 128;
constexpr int kGradBlocks = 296;  // 2 x 148 SMs
constexpr int kRowPad = 33;       // shared rows of 32 values, padded against bank conflicts

int fail(int code, const std::string& msg) {
  psl_detail_set_last_error(msg);
  return code;
}

#define TRAIN_CUDA(expr)                                                                               \
  do {                                                                                                 \
    cudaError_t e_ = (expr);                                                                           \
    if (e_ != cudaSuccess) return fail(PSL_ERR_CUDA, std::string(#expr) + ": " + cudaGetErrorString(e_)); \
  } while (0)

__device__ __forceinline__ uint32_t mix32(uint32_t x) {  // lowbias32 integer hash
  x ^= x >> 16;
  x *= 0x7feb352du;
  x ^= x >> 15;
  x *= 0x846ca68bu;
  x ^= x >> 16;
  return x;
}

struct GradShared {
  float w[kParams];
  float xn[kGradThreads][kMlpIn];
  float h1[kGradThreads][kRowPad];
  float h2[kGradThreads][kRowPad];
  float d1[kGradThreads][kRowPad];
  float d2[kGradThreads][kRowPad];
  float dz[kGradThreads];
  float loss[kGradThreads];
};

// Partial gradients of the batch samples [0, count): sample i is row first + i, or a
// hashed row of [0, n) when `random`.  partial[block][0..kTrainable) gets the block's
// gradient sums, partial[block][kTrainable] its loss sum.
__global__ void __launch_bounds__(kGradThreads) grad_kernel(const float* __restrict__ params, const float* __restrict__ X,
                                                            const float* __restrict__ T, long long n, long long first,
                                                            long long count, int random, uint32_t seed,
                                                            float* __restrict__ partial) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  GradShared& s = *reinterpret_cast<GradShared*>(smem_raw);
  for (int i = threadIdx.x; i < kParams; i += blockDim.x) s.w[i] = params[i];
  __syncthreads();
  const float inv_count = 1.f / (float)count;
  const float out_scale = s.w[kOutScale];
  constexpr int kPer = (kTrainable + kGradThreads - 1) / kGradThreads;
  float acc[kPer];
#pragma unroll
  for (int e = 0; e < kPer; ++e) acc[e] = 0.f;
  float loss = 0.f;
  for (long long base = (long long)blockIdx.x * kGradThreads; base < count; base += (long long)gridDim.x * kGradThreads) {
    const long long i = base + threadIdx.x;
    const bool valid = i < count;
    float xn[kMlpIn];
    float t = 0.f;
    if (valid) {
      const long long row = random ? (long long)(mix32(seed ^ mix32((uint32_t)i * 2654435761u + (uint32_t)(i >> 32))) % (uint64_t)n)
                                   : first + i;
#pragma unroll
      for (int k = 0; k < kMlpIn; ++k) xn[k] = (X[row * kMlpIn + k] - s.w[kShift + k]) * s.w[kScale + k];
      t = T[row] / out_scale;
    } else {
#pragma unroll
      for (int k = 0; k < kMlpIn; ++k) xn[k] = 0.f;
    }
    // forward
    float a1[32], a2[32];
#pragma unroll 4
    for (int o = 0; o < 32; ++o) {
      float z = s.w[kB1 + o];
#pragma unroll
      for (int k = 0; k < kMlpIn; ++k) z = fmaf(s.w[kW1 + o * kMlpIn + k], xn[k], z);
      a1[o] = z;
    }
#pragma unroll 4
    for (int o = 0; o < 32; ++o) {
      float z = s.w[kB2 + o];
#pragma unroll
      for (int k = 0; k < 32; ++k) z = fmaf(s.w[kW2 + o * 32 + k], fmaxf(a1[k], 0.f), z);
      a2[o] = z;
    }
    float z = s.w[kB3];
#pragma unroll
    for (int k = 0; k < 32; ++k) z = fmaf(s.w[kW3 + k], fmaxf(a2[k], 0.f), z);
    const float y = z > 20.f ? z : log1pf(expf(z));
    const float r = valid ? y - t : 0.f;
    loss += r * r;
    const float dz = 2.f * r * inv_count / (1.f + expf(-fminf(z, 50.f)));
    // backward to the hidden layers
    float d2[32];
#pragma unroll
    for (int o = 0; o < 32; ++o) d2[o] = a2[o] > 0.f ? dz * s.w[kW3 + o] : 0.f;
#pragma unroll 4
    for (int k = 0; k < 32; ++k) {
      float g = 0.f;
#pragma unroll
      for (int o = 0; o < 32; ++o) g = fmaf(d2[o], s.w[kW2 + o * 32 + k], g);
      s.d1[threadIdx.x][k] = a1[k] > 0.f ? g : 0.f;
    }
#pragma unroll
    for (int k = 0; k < 32; ++k) {
      s.h1[threadIdx.x][k] = fmaxf(a1[k], 0.f);
      s.h2[threadIdx.x][k] = fmaxf(a2[k], 0.f);
      s.d2[threadIdx.x][k] = d2[k];
    }
#pragma unroll
    for (int k = 0; k < kMlpIn; ++k) s.xn[threadIdx.x][k] = xn[k];
    s.dz[threadIdx.x] = dz;
    __syncthreads();
    // weight gradients: each thread owns entries e = threadIdx.x + kGradThreads * j
#pragma unroll
    for (int j = 0; j < kPer; ++j) {
      const int e = threadIdx.x + kGradThreads * j;
      if (e >= kTrainable) break;
      float g = 0.f;
      if (e < kB1) {
        const int o = e / kMlpIn, k = e % kMlpIn;
        for (int b = 0; b < kGradThreads; ++b) g = fmaf(s.d1[b][o], s.xn[b][k], g);
      } else if (e < kW2) {
        const int o = e - kB1;
        for (int b = 0; b < kGradThreads; ++b) g += s.d1[b][o];
      } else if (e < kB2) {
        const int o = (e - kW2) / 32, k = (e - kW2) % 32;
        for (int b = 0; b < kGradThreads; ++b) g = fmaf(s.d2[b][o], s.h1[b][k], g);
      } else if (e < kW3) {
        const int o = e - kB2;
        for (int b = 0; b < kGradThreads; ++b) g += s.d2[b][o];
      } else if (e < kB3) {
        const int k = e - kW3;
        for (int b = 0; b < kGradThreads; ++b) g = fmaf(s.dz[b], s.h2[b][k], g);
      } else {
        for (int b = 0; b < kGradThreads; ++b) g += s.dz[b];
      }
      acc[j] += g;
    }
    __syncthreads();
  }
  float* out = partial + (size_t)blockIdx.x * (kTrainable + 1);
#pragma unroll
  for (int j = 0; j < kPer; ++j) {
    const int e = threadIdx.x + kGradThreads * j;
    if (e < kTrainable) out[e] = acc[j];
  }
  s.loss[threadIdx.x] = loss;
  __syncthreads();
  if (threadIdx.x == 0) {
    float l = 0.f;
    for (int b = 0; b < kGradThreads; ++b) l += s.loss[b];
    out[kTrainable] = l;
  }
}

// grad[e] = sum over blocks (in block order, FP64) of partial[block][e]; grad[kTrainable] is
// the mean loss.
__global__ void reduce_kernel(const float* __restrict__ partial, int blocks, long long count, double* __restrict__ grad) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e > kTrainable) return;
  double s = 0.0;
  for (int b = 0; b < blocks; ++b) s += (double)partial[(size_t)b * (kTrainable + 1) + e];
  grad[e] = e == kTrainable ? s / (double)count : s;
}

__global__ void adam_kernel(float* __restrict__ params, float* __restrict__ m, float* __restrict__ v,
                            const double* __restrict__ grad, float lr, float beta1, float beta2, float eps, int step) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= kTrainable) return;
  const float g = (float)grad[e];
  const float mm = beta1 * m[e] + (1.f - beta1) * g;
  const float vv = beta2 * v[e] + (1.f - beta2) * g * g;
  m[e] = mm;
  v[e] = vv;
  const float mh = mm / (1.f - powf(beta1, (float)step));
  const float vh = vv / (1.f - powf(beta2, (float)step));
  params[e] -= lr * mh / (sqrtf(vh) + eps);
}

// ---- samples from a fine periodic box ----
constexpr int kCoarseRecord = 19;  // 10 features, 3 filtered velocity, 6 subfilter stress

template <typename S>
__global__ void filter_kernel(GridView<S> fine, int fnx, int fny, int M, float* __restrict__ rec) {
  const long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (id >= (long long)M * M * M) return;
  const int I = (int)(id % M), J = (int)((id / M) % M), K = (int)(id / ((long long)M * M));
  float f[27];
#pragma unroll
  for (int q = 0; q < 27; ++q) f[q] = 0.f;
  float uu[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
  for (int c = 0; c < 8; ++c) {
    const int i = 2 * I + (c & 1), j = 2 * J + ((c >> 1) & 1), k = 2 * K + (c >> 2);
    const uint32_t cell = ((uint32_t)k * fny + j) * fnx + i;
    float fc[27];
    load_cell<S>(fine, cell, fc);
    float rho = 0.f, jx = 0.f, jy = 0.f, jz = 0.f;
#pragma unroll
    for (int q = 0; q < 27; ++q) {
      f[q] += fc[q];
      rho += fc[q];
      jx += cx(q) * fc[q];
      jy += cy(q) * fc[q];
      jz += cz(q) * fc[q];
    }
    const float ux = jx / rho, uy = jy / rho, uz = jz / rho;
    uu[0] += ux * ux;
    uu[1] += uy * uy;
    uu[2] += uz * uz;
    uu[3] += ux * uy;
    uu[4] += ux * uz;
    uu[5] += uy * uz;
  }
#pragma unroll
  for (int q = 0; q < 27; ++q) f[q] *= 0.125f;
  rescale(f, false);
  float Km[3][3][3];
  float rho, ux, uy, uz, inv_rho;
  central_moments(f, Km, rho, ux, uy, uz, inv_rho);
  float x[kMlpIn];
  mlp_features(Km[2][0][0], Km[0][2][0], Km[0][0][2], Km[1][1][0], Km[1][0][1], Km[0][1][1], rho, inv_rho, 1.f, x);
  float* r = rec + id * kCoarseRecord;
#pragma unroll
  for (int k = 0; k < kMlpIn; ++k) r[k] = x[k];
  r[10] = ux;
  r[11] = uy;
  r[12] = uz;
  r[13] = uu[0] * 0.125f - ux * ux;
  r[14] = uu[1] * 0.125f - uy * uy;
  r[15] = uu[2] * 0.125f - uz * uz;
  r[16] = uu[3] * 0.125f - ux * uy;
  r[17] = uu[4] * 0.125f - ux * uz;
  r[18] = uu[5] * 0.125f - uy * uz;
}

// Targets from the records (strain rate of the filtered velocity, periodic central
// differences) and the selected samples appended at X/T + `at`: cell `id` is selected when
// id % stride == phase.
__global__ void target_kernel(const float* __restrict__ rec, int M, int stride, int phase, float* __restrict__ X,
                              float* __restrict__ T, long long at) {
  const long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (id >= (long long)M * M * M || id % stride != phase) return;
  const int I = (int)(id % M), J = (int)((id / M) % M), K = (int)(id / ((long long)M * M));
  auto u = [&](int i, int j, int k, int comp) {
    i = (i + M) % M;
    j = (j + M) % M;
    k = (k + M) % M;
    return rec[(((long long)k * M + j) * M + i) * kCoarseRecord + 10 + comp];
  };
  float g[3][3];  // g[a][b] = d u_b / d x_a
  for (int b = 0; b < 3; ++b) {
    g[0][b] = 0.5f * (u(I + 1, J, K, b) - u(I - 1, J, K, b));
    g[1][b] = 0.5f * (u(I, J + 1, K, b) - u(I, J - 1, K, b));
    g[2][b] = 0.5f * (u(I, J, K + 1, b) - u(I, J, K - 1, b));
  }
  float Sm[3][3];
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) Sm[a][b] = 0.5f * (g[a][b] + g[b][a]);
  const float* r = rec + id * kCoarseRecord;
  const float tr = (r[13] + r[14] + r[15]) * (1.f / 3.f);
  const float tau[3][3] = {{r[13] - tr, r[16], r[17]}, {r[16], r[14] - tr, r[18]}, {r[17], r[18], r[15] - tr}};
  float ts = 0.f, ss = 0.f;
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) {
      ts += tau[a][b] * Sm[a][b];
      ss += Sm[a][b] * Sm[a][b];
    }
  const float nu_t = fmaxf(0.f, -ts / (2.f * ss + 1e-30f));
  const long long slot = at + id / stride;
#pragma unroll
  for (int k = 0; k < kMlpIn; ++k) X[slot * kMlpIn + k] = r[k];
  T[slot] = nu_t;
}

void to_flat(const psl_sgs_mlp& m, float* p) {
  std::memcpy(p + kW1, m.w1, sizeof(m.w1));
  std::memcpy(p + kB1, m.b1, sizeof(m.b1));
  std::memcpy(p + kW2, m.w2, sizeof(m.w2));
  std::memcpy(p + kB2, m.b2, sizeof(m.b2));
  std::memcpy(p + kW3, m.w3, sizeof(m.w3));
  p[kB3] = m.b3;
  std::memcpy(p + kShift, m.in_shift, sizeof(m.in_shift));
  std::memcpy(p + kScale, m.in_scale, sizeof(m.in_scale));
  p[kOutScale] = m.out_scale;
}

void from_flat(const float* p, psl_sgs_mlp& m) {
  std::memcpy(m.w1, p + kW1, sizeof(m.w1));
  std::memcpy(m.b1, p + kB1, sizeof(m.b1));
  std::memcpy(m.w2, p + kW2, sizeof(m.w2));
  std::memcpy(m.b2, p + kB2, sizeof(m.b2));
  std::memcpy(m.w3, p + kW3, sizeof(m.w3));
  m.b3 = p[kB3];
  std::memcpy(m.in_shift, p + kShift, sizeof(m.in_shift));
  std::memcpy(m.in_scale, p + kScale, sizeof(m.in_scale));
  m.out_scale = p[kOutScale];
}

}  // namespace

struct psl_sgs_trainer {
  int device = 0;
  cudaStream_t stream = nullptr;
  long long capacity = 0, count = 0;
  float* X = nullptr;  // [capacity][10] raw features
  float* T = nullptr;  // [capacity] targets
  float* params = nullptr;  // kParams
  float* m = nullptr;       // Adam moments (kTrainable each)
  float* v = nullptr;
  int step = 0;
  float* partial = nullptr;  // [kGradBlocks][kTrainable + 1]
  double* grad = nullptr;    // kTrainable + 1
};

namespace {

int run_gradient(psl_sgs_trainer* t, long long first, long long count, int random, uint32_t seed) {
  const size_t smem = sizeof(GradShared);
  TRAIN_CUDA(cudaFuncSetAttribute(grad_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const int blocks = (int)std::min<long long>(kGradBlocks, (count + kGradThreads - 1) / kGradThreads);
  grad_kernel<<<blocks, kGradThreads, smem, t->stream>>>(t->params, t->X, t->T, t->count, first, count, random, seed,
                                                         t->partial);
  reduce_kernel<<<(kTrainable + 1 + 255) / 256, 256, 0, t->stream>>>(t->partial, blocks, count, t->grad);
  TRAIN_CUDA(cudaGetLastError());
  return PSL_OK;
}

}  // namespace

int psl_sgs_trainer_create(long long capacity, psl_sgs_trainer** out) {
  if (!out || capacity <= 0) return fail(PSL_ERR_INVALID, "psl_sgs_trainer_create: bad argument");
  *out = nullptr;
  int ndev = 0;
  TRAIN_CUDA(cudaGetDeviceCount(&ndev));
  if (ndev <= 0) return fail(PSL_ERR_CUDA, "psl_sgs_trainer_create: no CUDA device");
  psl_sgs_trainer* t = new psl_sgs_trainer();
  cudaGetDevice(&t->device);
  t->capacity = capacity;
  cudaError_t e = cudaStreamCreateWithFlags(&t->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaMalloc(&t->X, (size_t)capacity * kMlpIn * sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc(&t->T, (size_t)capacity * sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc(&t->params, kParams * sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc(&t->m, kTrainable * sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc(&t->v, kTrainable * sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc(&t->partial, (size_t)kGradBlocks * (kTrainable + 1) * sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc(&t->grad, (kTrainable + 1) * sizeof(double));
  if (e == cudaSuccess) e = cudaMemset(t->params, 0, kParams * sizeof(float));
  if (e == cudaSuccess) e = cudaMemset(t->m, 0, kTrainable * sizeof(float));
  if (e == cudaSuccess) e = cudaMemset(t->v, 0, kTrainable * sizeof(float));
  if (e != cudaSuccess) {
    const std::string msg = std::string("psl_sgs_trainer_create: ") + cudaGetErrorString(e);
    cudaGetLastError();
    psl_sgs_trainer_destroy(t);
    return fail(e == cudaErrorMemoryAllocation ? PSL_ERR_NOMEM : PSL_ERR_CUDA, msg);
  }
  *out = t;
  return PSL_OK;
}

int psl_sgs_trainer_destroy(psl_sgs_trainer* t) {
  if (!t) return PSL_OK;
  DeviceGuard dg(t->device);
  if (t->stream) cudaStreamSynchronize(t->stream);
  for (void* p : {(void*)t->X, (void*)t->T, (void*)t->params, (void*)t->m, (void*)t->v, (void*)t->partial, (void*)t->grad})
    if (p) cudaFree(p);
  if (t->stream) cudaStreamDestroy(t->stream);
  delete t;
  return PSL_OK;
}

int psl_sgs_trainer_clear(psl_sgs_trainer* t) {
  if (!t) return fail(PSL_ERR_INVALID, "psl_sgs_trainer_clear: null trainer");
  t->count = 0;
  return PSL_OK;
}

int psl_sgs_trainer_count(const psl_sgs_trainer* t, long long* count) {
  if (!t || !count) return fail(PSL_ERR_INVALID, "psl_sgs_trainer_count: null argument");
  *count = t->count;
  return PSL_OK;
}

int psl_sgs_trainer_add_samples(psl_sgs_trainer* t, const float* features, const float* targets, long long n) {
  if (!t || !features || !targets || n < 0) return fail(PSL_ERR_INVALID, "psl_sgs_trainer_add_samples: bad argument");
  if (t->count + n > t->capacity) return fail(PSL_ERR_INVALID, "psl_sgs_trainer_add_samples: capacity exceeded");
  DeviceGuard dg(t->device);
  TRAIN_CUDA(cudaMemcpyAsync(t->X + t->count * kMlpIn, features, (size_t)n * kMlpIn * sizeof(float),
                             cudaMemcpyHostToDevice, t->stream));
  TRAIN_CUDA(cudaMemcpyAsync(t->T + t->count, targets, (size_t)n * sizeof(float), cudaMemcpyHostToDevice, t->stream));
  TRAIN_CUDA(cudaStreamSynchronize(t->stream));
  t->count += n;
  return PSL_OK;
}

int psl_sgs_trainer_get_samples(psl_sgs_trainer* t, long long first, long long n, float* features, float* targets) {
  if (!t || first < 0 || n < 0 || first + n > t->count) return fail(PSL_ERR_INVALID, "psl_sgs_trainer_get_samples: bad range");
  DeviceGuard dg(t->device);
  if (features)
    TRAIN_CUDA(cudaMemcpyAsync(features, t->X + first * kMlpIn, (size_t)n * kMlpIn * sizeof(float),
                               cudaMemcpyDeviceToHost, t->stream));
  if (targets)
    TRAIN_CUDA(cudaMemcpyAsync(targets, t->T + first, (size_t)n * sizeof(float), cudaMemcpyDeviceToHost, t->stream));
  TRAIN_CUDA(cudaStreamSynchronize(t->stream));
  return PSL_OK;
}

int psl_sgs_trainer_add_filtered(psl_sgs_trainer* t, psl_grid* fine, int M, int stride, unsigned int phase) {
  if (!t || !fine || M < 2 || stride < 1) return fail(PSL_ERR_INVALID, "psl_sgs_trainer_add_filtered: bad argument");
  const psl_info& I = fine->info;
  if (I.cell_count_x != 2 * M + 1 || I.cell_count_y != 2 * M + 1 || I.cell_count_z != 2 * M)
    return fail(PSL_ERR_INVALID, "psl_sgs_trainer_add_filtered: fine grid must be (2M+1) x (2M+1) x 2M (periodic box)");
  if (fine->storage == kStoreF64) return fail(PSL_ERR_INVALID, "psl_sgs_trainer_add_filtered: FP64 storage");
  const long long cells = (long long)M * M * M;
  const long long selected = (cells - (long long)(phase % stride) + stride - 1) / stride;
  if (t->count + selected > t->capacity) return fail(PSL_ERR_INVALID, "psl_sgs_trainer_add_filtered: capacity exceeded");
  DeviceGuard dg(t->device);
  float* rec = nullptr;
  TRAIN_CUDA(cudaMalloc(&rec, (size_t)cells * kCoarseRecord * sizeof(float)));
  TRAIN_CUDA(cudaStreamSynchronize(fine->stream));
  const unsigned int nb = (unsigned int)((cells + 255) / 256);
  auto go = [&](auto s) {
    using S = decltype(s);
    GridView<S> v;
    typename S::type* base = static_cast<typename S::type*>(fine->f);
    for (int q = 0; q < 27; ++q) {
      v.fq[q] = base + (size_t)q * fine->f_stride;
      v.shift[q] = fine->shift[q];
    }
    v.n = fine->n;
    filter_kernel<S><<<nb, 256, 0, t->stream>>>(v, I.cell_count_x, I.cell_count_y, M, rec);
  };
  switch (fine->storage) {
    case kStoreF32: go(StoreF32{}); break;
    case kStoreF16: go(StoreF16{}); break;
    default: go(StoreBF16{}); break;
  }
  target_kernel<<<nb, 256, 0, t->stream>>>(rec, M, stride, (int)(phase % stride), t->X, t->T, t->count);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaStreamSynchronize(t->stream);
  cudaFree(rec);
  if (e != cudaSuccess) return fail(PSL_ERR_CUDA, std::string("psl_sgs_trainer_add_filtered: ") + cudaGetErrorString(e));
  t->count += selected;
  return PSL_OK;
}

int psl_sgs_trainer_set_params(psl_sgs_trainer* t, const psl_sgs_mlp* mlp) {
  if (!t || !mlp) return fail(PSL_ERR_INVALID, "psl_sgs_trainer_set_params: null argument");
  DeviceGuard dg(t->device);
  std::vector<float> p(kParams);
  to_flat(*mlp, p.data());
  TRAIN_CUDA(cudaMemcpyAsync(t->params, p.data(), kParams * sizeof(float), cudaMemcpyHostToDevice, t->stream));
  TRAIN_CUDA(cudaMemsetAsync(t->m, 0, kTrainable * sizeof(float), t->stream));
  TRAIN_CUDA(cudaMemsetAsync(t->v, 0, kTrainable * sizeof(float), t->stream));
  TRAIN_CUDA(cudaStreamSynchronize(t->stream));
  t->step = 0;
  return PSL_OK;
}

int psl_sgs_trainer_get_params(psl_sgs_trainer* t, psl_sgs_mlp* mlp) {
  if (!t || !mlp) return fail(PSL_ERR_INVALID, "psl_sgs_trainer_get_params: null argument");
  DeviceGuard dg(t->device);
  std::vector<float> p(kParams);
  TRAIN_CUDA(cudaMemcpyAsync(p.data(), t->params, kParams * sizeof(float), cudaMemcpyDeviceToHost, t->stream));
  TRAIN_CUDA(cudaStreamSynchronize(t->stream));
  from_flat(p.data(), *mlp);
  return PSL_OK;
}

int psl_sgs_trainer_gradient(psl_sgs_trainer* t, long long first, long long count, psl_sgs_mlp* grad, double* loss) {
  if (!t || first < 0 || count <= 0 || first + count > t->count)
    return fail(PSL_ERR_INVALID, "psl_sgs_trainer_gradient: bad range");
  DeviceGuard dg(t->device);
  int rc = run_gradient(t, first, count, 0, 0);
  if (rc) return rc;
  std::vector<double> g(kTrainable + 1);
  TRAIN_CUDA(cudaMemcpyAsync(g.data(), t->grad, (kTrainable + 1) * sizeof(double), cudaMemcpyDeviceToHost, t->stream));
  TRAIN_CUDA(cudaStreamSynchronize(t->stream));
  if (grad) {
    std::vector<float> p(kParams, 0.f);
    for (int e = 0; e < kTrainable; ++e) p[e] = (float)g[e];
    from_flat(p.data(), *grad);
  }
  if (loss) *loss = g[kTrainable];
  return PSL_OK;
}

int psl_sgs_trainer_train(psl_sgs_trainer* t, int steps, int batch, float lr, unsigned int seed, double* last_loss) {
  if (!t || steps < 0 || batch <= 0 || t->count <= 0) return fail(PSL_ERR_INVALID, "psl_sgs_trainer_train: bad argument");
  DeviceGuard dg(t->device);
  for (int s = 0; s < steps; ++s) {
    ++t->step;
    int rc = run_gradient(t, 0, batch, 1, seed * 0x9e3779b9u + (uint32_t)t->step);
    if (rc) return rc;
    adam_kernel<<<(kTrainable + 255) / 256, 256, 0, t->stream>>>(t->params, t->m, t->v, t->grad, lr, 0.9f, 0.999f,
                                                                  1e-8f, t->step);
  }
  TRAIN_CUDA(cudaGetLastError());
  if (last_loss) {
    TRAIN_CUDA(cudaMemcpyAsync(last_loss, t->grad + kTrainable, sizeof(double), cudaMemcpyDeviceToHost, t->stream));
  }
  TRAIN_CUDA(cudaStreamSynchronize(t->stream));
  return PSL_OK;
}
