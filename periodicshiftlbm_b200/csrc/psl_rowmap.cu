// Population rows mapped twice in virtual memory.
//
// A periodic-shift row is a ring of N values: cell c of population q lives at
// (c + shift_q) mod N (applyStreaming.h:9-27 moves shift_q instead of the data).  When the
// row's physical memory is mapped at two consecutive virtual ranges, [R, R + N) and
// [R + N, R + 2N) show the same values, so the update can address c + shift_q < 2N
// directly: no per-population wrap compare in the kernels that read every population of
// every cell.  The second mapping costs virtual address space only.
//
// Needs the CUDA driver's virtual-memory management (cuMemCreate / cuMemMap), reached
// through cudaGetDriverEntryPoint so that the library does not link libcuda itself, and a
// row size that is a whole number of the allocation granularity (2 MiB on current GPUs:
// 1,048,576 FP16 cells, 524,288 FP32 cells).  Other grids keep one plain allocation.
#include <cuda.h>
#include <cuda_runtime.h>

#include <mutex>
#include <string>
#include <vector>

#include "psl_rowmap.h"

namespace {

struct DriverVmm {
  decltype(&cuMemGetAllocationGranularity) granularity = nullptr;
  decltype(&cuMemCreate) create = nullptr;
  decltype(&cuMemRelease) release = nullptr;
  decltype(&cuMemAddressReserve) reserve = nullptr;
  decltype(&cuMemAddressFree) address_free = nullptr;
  decltype(&cuMemMap) map = nullptr;
  decltype(&cuMemUnmap) unmap = nullptr;
  decltype(&cuMemSetAccess) set_access = nullptr;
  bool ok = false;
};

template <typename Fn>
bool entry(const char* name, Fn* fn) {
  void* p = nullptr;
  cudaDriverEntryPointQueryResult status = cudaDriverEntryPointSymbolNotFound;
  if (cudaGetDriverEntryPoint(name, &p, cudaEnableDefault, &status) != cudaSuccess ||
      status != cudaDriverEntryPointSuccess || !p) {
    cudaGetLastError();
    return false;
  }
  *fn = reinterpret_cast<Fn>(p);
  return true;
}

const DriverVmm& driver() {
  static DriverVmm d;
  static std::once_flag once;
  std::call_once(once, [] {
    d.ok = entry("cuMemGetAllocationGranularity", &d.granularity) && entry("cuMemCreate", &d.create) &&
           entry("cuMemRelease", &d.release) && entry("cuMemAddressReserve", &d.reserve) &&
           entry("cuMemAddressFree", &d.address_free) && entry("cuMemMap", &d.map) &&
           entry("cuMemUnmap", &d.unmap) && entry("cuMemSetAccess", &d.set_access);
  });
  return d;
}

CUmemAllocationProp device_prop(int device) {
  CUmemAllocationProp prop = {};
  prop.type = CU_MEM_ALLOCATION_TYPE_PINNED;
  prop.location.type = CU_MEM_LOCATION_TYPE_DEVICE;
  prop.location.id = device;
  return prop;
}

}  // namespace

struct psl_row_map {
  const DriverVmm* drv = nullptr;
  CUdeviceptr base = 0;
  size_t reserved = 0;   // bytes of virtual address space (2 x rows x row_bytes)
  size_t row_bytes = 0;
  int mappings = 0;      // ranges of row_bytes mapped so far, in address order from base
  std::vector<CUmemGenericAllocationHandle> handles;
};

void psl_row_map_destroy(psl_row_map* m) {
  if (!m) return;
  const DriverVmm& d = *m->drv;
  for (int i = 0; i < m->mappings; ++i) d.unmap(m->base + (size_t)i * m->row_bytes, m->row_bytes);
  for (CUmemGenericAllocationHandle h : m->handles) d.release(h);
  if (m->reserved) d.address_free(m->base, m->reserved);
  delete m;
}

cudaError_t psl_row_map_create(int device, size_t row_bytes, int rows, void** base, psl_row_map** out,
                               std::string* why) {
  *base = nullptr;
  *out = nullptr;
  const DriverVmm& d = driver();
  if (!d.ok) {
    if (why) *why = "the driver has no virtual-memory management entry points";
    return cudaErrorNotSupported;
  }
  const CUmemAllocationProp prop = device_prop(device);
  size_t gran = 0;
  if (d.granularity(&gran, &prop, CU_MEM_ALLOC_GRANULARITY_MINIMUM) != CUDA_SUCCESS || gran == 0) {
    if (why) *why = "cuMemGetAllocationGranularity failed";
    return cudaErrorNotSupported;
  }
  if (row_bytes == 0 || row_bytes % gran != 0 || rows <= 0) {
    if (why) *why = "row size " + std::to_string(row_bytes) + " is not a multiple of " + std::to_string(gran);
    return cudaErrorNotSupported;
  }
  psl_row_map* m = new psl_row_map();
  m->drv = &d;
  const size_t total = 2 * row_bytes * (size_t)rows;
  if (d.reserve(&m->base, total, gran, 0, 0) != CUDA_SUCCESS) {
    if (why) *why = "cuMemAddressReserve failed";
    delete m;
    return cudaErrorMemoryAllocation;
  }
  m->reserved = total;
  m->row_bytes = row_bytes;
  CUmemAccessDesc access = {};
  access.location = prop.location;
  access.flags = CU_MEM_ACCESS_FLAGS_PROT_READWRITE;
  for (int r = 0; r < rows; ++r) {
    CUmemGenericAllocationHandle h = 0;
    const CUresult rc = d.create(&h, row_bytes, &prop, 0);
    if (rc != CUDA_SUCCESS) {
      if (why) *why = "cuMemCreate failed";
      psl_row_map_destroy(m);
      return rc == CUDA_ERROR_OUT_OF_MEMORY ? cudaErrorMemoryAllocation : cudaErrorUnknown;
    }
    m->handles.push_back(h);
    for (int copy = 0; copy < 2; ++copy) {
      const CUdeviceptr at = m->base + (2 * (size_t)r + copy) * row_bytes;
      if (d.map(at, row_bytes, 0, h, 0) != CUDA_SUCCESS) {
        if (why) *why = "cuMemMap failed";
        psl_row_map_destroy(m);
        return cudaErrorUnknown;
      }
      ++m->mappings;
      if (d.set_access(at, row_bytes, &access, 1) != CUDA_SUCCESS) {
        if (why) *why = "cuMemSetAccess failed";
        psl_row_map_destroy(m);
        return cudaErrorUnknown;
      }
    }
  }
  *base = reinterpret_cast<void*>(m->base);
  *out = m;
  return cudaSuccess;
}
