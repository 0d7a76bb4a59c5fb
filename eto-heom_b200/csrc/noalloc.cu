// Delay scan for callers that may not allocate device memory.
//
// heom_run_scan_device needs a plan, and a plan allocates (tables, work queue, point
// ordering).  Some callers cannot let a library allocate: a service that reserves its
// whole device-memory budget at start-up (its own pool, or an ML framework's caching
// allocator, holds everything) and must not see cudaMalloc fail or stall later, or an
// application that only permits allocation during initialisation.  This entry point
// takes the problem from the host handle and the caller's device buffers and keeps its
// own scratch -- the work-queue counter, the point ordering and the packed hierarchy
// tables and system matrices -- in one file-scope __device__ array of fixed size, so it
// performs no device allocation at all.
//
// Limits and sharing:
//  * the array is kNoAllocScratchBytes (4 MiB) on every GPU that loads the library and
//    stays allocated until the process exits;
//  * at most kNoAllocMaxPoints points per call, and the packed tables of the problem
//    must fit beside them; larger requests fail with HEOM_ERR_CAPACITY;
//  * every call on a device reuses the same array and leaves the last call's contents
//    in it; the work-queue counter is cleared at the start of every call on the stream.
//    Calls whose work overlaps on the GPU (different streams, or different host threads
//    without ordering) race on the array and must be serialised by the caller;
//  * the first call on a device resolves the array's device address
//    (cudaGetSymbolAddress) with that device current; make that first call before any
//    stream capture on that device.
#include <cuda_runtime.h>

#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/heom.h"
#include "heom_host.h"
#include "scan.h"

namespace {

constexpr size_t kNoAllocScratchBytes = 4u << 20;
constexpr int kNoAllocMaxPoints = 65536;
constexpr size_t kCounterBytes = 256;
constexpr int kMaxDevices = 64;

__device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

std::mutex g_mu;
unsigned char *g_base[kMaxDevices] = {};

size_t align256(size_t v) { return (v + 255) & ~(size_t)255; }

// Device address of the scratch array on the current device (once per device).
int scratch_base(int dev, unsigned char **out) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_base[dev]) {
    void *ptr = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
    if (e != cudaSuccess)
      return heom::set_error(HEOM_ERR_CUDA, std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e));
    g_base[dev] = (unsigned char *)ptr;
  }
  *out = g_base[dev];
  return HEOM_OK;
}

} // namespace

extern "C" int heom_run_scan_noalloc(const heom_problem *prob, int precision, const heom_scan_point *d_pts, int n,
                                     double *d_P, const long long *d_offsets, void *stream) {
  if (!prob || n < 0 || (n > 0 && (!d_pts || !d_P || !d_offsets)))
    return heom::set_error(HEOM_ERR_ARG, "bad argument");
  if (prob->p.dynamics) return heom::set_error(HEOM_ERR_UNSUPPORTED, "population-dynamics keys have no delay scan");
  if (precision != HEOM_FP32_BULK && precision != HEOM_FP64)
    return heom::set_error(HEOM_ERR_ARG, "heom_run_scan_noalloc takes HEOM_FP32_BULK or HEOM_FP64");
  if (n > kNoAllocMaxPoints)
    return heom::set_error(HEOM_ERR_CAPACITY, "heom_run_scan_noalloc: " + std::to_string(n) +
                                                  " points exceed the limit of " + std::to_string(kNoAllocMaxPoints) +
                                                  " per call");
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return heom::set_error(HEOM_ERR_CUDA, std::string("no CUDA device: ") + cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices) return heom::set_error(HEOM_ERR_UNSUPPORTED, "device ordinal above 63");
  unsigned char *base = nullptr;
  int rc = scratch_base(dev, &base);
  if (rc) return rc;

  heom_dev::ScanState s;
  std::vector<unsigned char> tables;
  if (!heom_dev::scan_prepare(s, prob->p, precision, n > 0 ? n : 1, tables))
    return heom::set_error(HEOM_ERR_UNSUPPORTED, "scan path unavailable for this problem: " + s.why);
  std::vector<double> sys;
  heom_dev::scan_system_host(prob->p, sys);
  // layout: [counter][order: int per point][tables][system]
  const size_t off_order = kCounterBytes;
  const size_t off_tables = align256(off_order + sizeof(int) * (size_t)kNoAllocMaxPoints);
  const size_t off_sys = align256(off_tables + tables.size());
  const size_t need = off_sys + sizeof(double) * sys.size();
  if (need > kNoAllocScratchBytes)
    return heom::set_error(HEOM_ERR_CAPACITY, "heom_run_scan_noalloc: the problem's tables need " +
                                                  std::to_string(need) + " bytes of the " +
                                                  std::to_string(kNoAllocScratchBytes) + "-byte static scratch");
  if (n == 0) return HEOM_OK;
  cudaStream_t st = (cudaStream_t)stream;
  s.d_counter = (int *)base;
  s.d_order = (int *)(base + off_order);
  s.d_tables = base + off_tables;
  s.d_sys = (double *)(base + off_sys);
  e = cudaMemcpyAsync(s.d_tables, tables.data(), tables.size(), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(s.d_sys, sys.data(), sizeof(double) * sys.size(), cudaMemcpyHostToDevice, st);
  if (e != cudaSuccess) return heom::set_error(HEOM_ERR_CUDA, std::string("scratch upload: ") + cudaGetErrorString(e));
  // the order kernel (or the reset kernel for unsorted batches) clears the counter first
  e = heom_dev::scan_enqueue(s, d_pts, n, d_P, d_offsets, st);
  if (e != cudaSuccess) return heom::set_error(HEOM_ERR_CUDA, std::string("scan launch: ") + cudaGetErrorString(e));
  return HEOM_OK;
}
