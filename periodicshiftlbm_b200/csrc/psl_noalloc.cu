// Momentum-exchange force without any device allocation.
//
// psl_sphere_force (psl_capi.cu) keeps its per-block partial sums in scratch memory that
// psl_grid_create allocates.  Some callers cannot allocate device memory when they need
// the force: code that runs its step loop inside CUDA stream capture (cudaMalloc and
// cudaFree are not stream operations and cudaFree synchronises the device), applications
// whose device memory belongs to another allocator's pool (a framework caching allocator
// or a fixed budget carved out at start-up), and real-time loops that must not block on
// an allocation.  psl_momentum_exchange_force_noalloc serves them: it reads populations
// and markers from the caller's own device buffers, writes the force to the caller's device
// buffer, and keeps its partial sums in the fixed array below, which every GPU that loads
// this library holds until the process exits.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "psl.h"
#include "psl_kernels.cuh"

using namespace psl;

namespace {

constexpr int kNoAllocBlocks = 1024;          // partial sums the fixed scratch holds
constexpr int kNoAllocThreads = 256;          // threads per block of the partial-sum kernel
constexpr long long kNoAllocCellsPerBlock = 4096;
// Largest box accepted: kNoAllocBlocks blocks of kNoAllocCellsPerBlock cells (4,194,304).
constexpr long long kNoAllocMaxBoxCells = kNoAllocBlocks * kNoAllocCellsPerBlock;
constexpr int kMaxDevices = 64;

// 1024 x 3 partials + 3 spare doubles: 24.6 KB per device.
static __device__ __align__(256) double psl_noalloc_force_scratch[kNoAllocBlocks * 3 + 3];

// Device address of the scratch array per device (scratch_on_current_device).  In host code
// the array's name is only a host-side stand-in, never a device address.
double* g_scratch[kMaxDevices] = {};
std::mutex g_scratch_mutex;

}  // namespace

// Defined in psl_capi.cu: sets the message psl_last_error() returns on this thread.
__attribute__((visibility("hidden"))) void psl_detail_set_last_error(const std::string& msg);

namespace {

int noalloc_fail(int code, const std::string& msg) {
  psl_detail_set_last_error(msg);
  return code;
}

// The scratch array's device address on the current device.  Outside stream capture it is
// looked up on every call (a device reset reloads the module, and a cached address would go
// stale); during capture, where a lookup could load the module inside the capture, the
// address of the last call outside capture is used.
int scratch_on_current_device(cudaStream_t stream, double** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return noalloc_fail(PSL_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices) return noalloc_fail(PSL_ERR_CUDA, "device ordinal out of range");
  cudaStreamCaptureStatus capture = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(stream, &capture) != cudaSuccess) {
    cudaGetLastError();
    capture = cudaStreamCaptureStatusActive;  // status unknown: do not touch the module
  }
  std::lock_guard<std::mutex> lock(g_scratch_mutex);
  if (capture == cudaStreamCaptureStatusNone || !g_scratch[dev]) {
    double* p = nullptr;
    e = cudaGetSymbolAddress((void**)&p, psl_noalloc_force_scratch);
    if (e != cudaSuccess || !p)
      return noalloc_fail(PSL_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e) +
                                            (capture == cudaStreamCaptureStatusNone
                                                 ? ""
                                                 : " (first call inside stream capture: make one call outside "
                                                   "capture first)"));
    g_scratch[dev] = p;
  }
  *out = g_scratch[dev];
  return PSL_OK;
}

}  // namespace

int psl_momentum_exchange_force_noalloc(const float* populations, long long row_stride, const int* shifts27,
                                        long long cell_count, const uint8_t* markers, int nx, int ny, int nz,
                                        const int* box_lo3, const int* box_hi3, double* force3, void* cuda_stream) {
  if (!populations || !shifts27 || !markers || !box_lo3 || !box_hi3 || !force3)
    return noalloc_fail(PSL_ERR_INVALID, "psl_momentum_exchange_force_noalloc: null argument");
  if (nx <= 0 || ny <= 0 || nz <= 0 || cell_count != (long long)nx * ny * nz || cell_count >= (1LL << 31))
    return noalloc_fail(PSL_ERR_INVALID, "psl_momentum_exchange_force_noalloc: cell_count must equal nx*ny*nz < 2^31");
  if (row_stride < cell_count)
    return noalloc_fail(PSL_ERR_INVALID, "psl_momentum_exchange_force_noalloc: row_stride smaller than cell_count");
  for (int q = 0; q < 27; ++q)
    if (shifts27[q] < 0 || shifts27[q] >= cell_count)
      return noalloc_fail(PSL_ERR_INVALID, "psl_momentum_exchange_force_noalloc: shift outside [0, cell_count)");
  const int dims[3] = {nx, ny, nz};
  long long cells = 1;
  for (int a = 0; a < 3; ++a) {
    if (box_lo3[a] < 0 || box_hi3[a] > dims[a] || box_hi3[a] < box_lo3[a])
      return noalloc_fail(PSL_ERR_INVALID, "psl_momentum_exchange_force_noalloc: box outside the grid");
    cells *= box_hi3[a] - box_lo3[a];
  }
  if (cells > kNoAllocMaxBoxCells)
    return noalloc_fail(PSL_ERR_INVALID,
                        "psl_momentum_exchange_force_noalloc: box has " + std::to_string(cells) +
                            " cells, more than the fixed scratch serves (" + std::to_string(kNoAllocMaxBoxCells) + ")");
  cudaStream_t stream = static_cast<cudaStream_t>(cuda_stream);
  double* scratch = nullptr;
  const int rc = scratch_on_current_device(stream, &scratch);
  if (rc != PSL_OK) return rc;
  GridView<StoreF32> g;
  for (int q = 0; q < 27; ++q) {
    g.fq[q] = const_cast<float*>(populations) + (size_t)q * (size_t)row_stride;
    g.shift[q] = (uint32_t)shifts27[q];
  }
  g.n = (uint32_t)cell_count;
  // Every block writes its own partial before the final kernel reads it, so the scratch
  // needs no clearing between calls.
  const int nb = cells == 0 ? 1 : (int)((cells + kNoAllocCellsPerBlock - 1) / kNoAllocCellsPerBlock);
  force_partial_kernel<StoreF32><<<nb, kNoAllocThreads, 0, stream>>>(
      g, markers, nx, ny, box_lo3[0], box_lo3[1], box_lo3[2], box_hi3[0] - box_lo3[0], box_hi3[1] - box_lo3[1],
      box_hi3[2] - box_lo3[2], scratch);
  force_final_kernel<<<1, 256, 0, stream>>>(scratch, nb, force3);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess)
    return noalloc_fail(PSL_ERR_CUDA, std::string("psl_momentum_exchange_force_noalloc: ") + cudaGetErrorString(e));
  return PSL_OK;
}
