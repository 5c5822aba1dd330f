// noalloc.cu -- max |a[i]| without any device allocation.
//
// pf5d_abs_max keeps its block partial maxima in a workspace it allocates
// with cudaMalloc the first time it runs on a device.  Some callers cannot
// let a library do that: a host that has handed the whole GPU to its own
// memory pool and forbids other allocations, a loop that must never hit the
// device-wide synchronisation cudaMalloc/cudaFree can cause, or code running
// where CUDA allocation calls are not permitted.  pf5d_abs_max_noalloc gives
// them the same reduction with its scratch in a statically sized
// __device__ array that the CUDA runtime creates when it loads this library
// on a device, so the call itself allocates nothing.
//
// Same result as pf5d_abs_max: the maximum of |a[i]| starting from 0.0, NaN
// entries ignored (phasefield5d/solver/operators.py:161-175 semantics); the
// maximum of a set of doubles does not depend on the order it is taken in.
#include <mutex>

#include "pf5d_device.cuh"
#include "pf5d_host.h"

namespace pf5d {
namespace {

constexpr int kNoAllocThreads = 256;
constexpr int kNoAllocPerThread = 8;
constexpr int64_t kNoAllocPerBlock = (int64_t)kNoAllocThreads * kNoAllocPerThread;  // 2048
constexpr int kNoAllocPartials = 32768;                                              // 256 KiB

// One partial maximum per block of 2048 elements.  Every GPU that loads the
// library holds these 256 KiB until the process exits.  All calls share
// them: each call overwrites the partials it uses before reading them, so
// nothing has to be cleared between calls, but two calls whose kernels
// overlap on the GPU (different streams, no ordering) race on this array.
static __device__ __align__(256) double g_noalloc_partials[kNoAllocPartials];

__global__ void k_noalloc_partial(const double *__restrict__ a, int64_t n, double *partials) {
  __shared__ double red[kNoAllocThreads / 32];
  const int64_t base = blockIdx.x * kNoAllocPerBlock;
  double m = 0.0;
#pragma unroll
  for (int k = 0; k < kNoAllocPerThread; ++k) {
    const int64_t i = base + (int64_t)k * kNoAllocThreads + threadIdx.x;
    if (i < n) {
      const double v = fabs(a[i]);
      if (v > m) m = v;
    }
  }
  m = block_max<kNoAllocThreads>(m, red);
  if (threadIdx.x == 0) partials[blockIdx.x] = m;
}

__global__ void k_noalloc_final(const double *__restrict__ partials, int nparts, double *result) {
  __shared__ double red[kNoAllocThreads / 32];
  double m = 0.0;
  for (int i = threadIdx.x; i < nparts; i += kNoAllocThreads) m = fmax(m, partials[i]);
  m = block_max<kNoAllocThreads>(m, red);
  if (threadIdx.x == 0) *result = m;
}

// Device address of g_noalloc_partials, looked up once per device.  In host
// code the array's name only stands for the symbol; the kernels must be
// given the address cudaGetSymbolAddress returns while that device is
// current.
std::mutex g_addr_mutex;
double *g_addr[64] = {nullptr};

pf5d_status partials_address(double **out) {
  int dev = 0;
  PF5D_CUDA(cudaGetDevice(&dev));
  PF5D_REQUIRE(dev >= 0 && dev < 64, PF5D_ERR_ARG, "device ordinal %d out of range", dev);
  std::lock_guard<std::mutex> lock(g_addr_mutex);
  if (!g_addr[dev]) {
    void *p = nullptr;
    PF5D_CUDA(cudaGetSymbolAddress(&p, g_noalloc_partials));
    g_addr[dev] = static_cast<double *>(p);
  }
  *out = g_addr[dev];
  return PF5D_OK;
}

}  // namespace
}  // namespace pf5d

using namespace pf5d;

extern "C" pf5d_status pf5d_abs_max_noalloc(const double *a, int64_t n, double *result,
                                            void *stream) {
  PF5D_REQUIRE(result && n >= 0 && (a || n == 0), PF5D_ERR_ARG, "bad arguments");
  PF5D_REQUIRE(n <= (int64_t)kNoAllocPartials * kNoAllocPerBlock, PF5D_ERR_CAPACITY,
               "pf5d_abs_max_noalloc handles at most %lld elements (got %lld); use pf5d_abs_max",
               (long long)kNoAllocPartials * kNoAllocPerBlock, (long long)n);
  double *partials = nullptr;
  pf5d_status st = partials_address(&partials);
  if (st != PF5D_OK) return st;
  const int nparts = n > 0 ? (int)((n + kNoAllocPerBlock - 1) / kNoAllocPerBlock) : 1;
  cudaStream_t s = as_stream(stream);
  k_noalloc_partial<<<nparts, kNoAllocThreads, 0, s>>>(a, n, partials);
  PF5D_LAUNCHED();
  k_noalloc_final<<<1, kNoAllocThreads, 0, s>>>(partials, nparts, result);
  PF5D_LAUNCHED();
  return PF5D_OK;
}
