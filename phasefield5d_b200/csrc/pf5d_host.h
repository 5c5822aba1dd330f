// pf5d_host.h -- host-side helpers shared by the library's translation units:
// error text, CUDA/cuFFT status checks and launch geometry.
#pragma once

#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <initializer_list>
#include <string>

#include <cuda_runtime.h>

#include "../../include/pf5d.h"

namespace pf5d {

void set_error(const char *fmt, ...);

inline cudaStream_t as_stream(void *s) { return reinterpret_cast<cudaStream_t>(s); }

// A kernel instance as profilers print it, "name<a, b, ...>" (bools as 0/1),
// so reports can name the exact kernels a variant launches.
inline std::string kname(const char *name, std::initializer_list<long long> targs) {
  std::string s = name;
  s += "<";
  bool first = true;
  for (long long v : targs) {
    if (!first) s += ", ";
    s += std::to_string(v);
    first = false;
  }
  return s + ">";
}

// Number of SMs on the current device (cached per device).
int sm_count();

// Grid size for grid-stride element kernels: a multiple of the SM count.
inline unsigned grid_for(int64_t n, int threads, int waves = 8) {
  const int64_t want = (n + threads - 1) / threads;
  const int64_t cap = (int64_t)sm_count() * waves;
  return (unsigned)(want < 1 ? 1 : (want < cap ? want : cap));
}

// Launch with programmatic stream serialization: the kernel's grid may be
// scheduled while the previous kernel in the stream finishes; the kernel
// must call pdl_wait() before touching memory that kernel writes.
template <typename... KArgs, typename... Args>
cudaError_t launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem,
                       cudaStream_t s, Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kernel, args...);
}

}  // namespace pf5d

#define PF5D_CUDA(call)                                                             \
  do {                                                                              \
    cudaError_t e_ = (call);                                                        \
    if (e_ != cudaSuccess) {                                                        \
      pf5d::set_error("%s:%d %s: %s", __FILE__, __LINE__, #call, cudaGetErrorString(e_)); \
      return PF5D_ERR_CUDA;                                                         \
    }                                                                               \
  } while (0)

#define PF5D_LAUNCHED()                                                             \
  do {                                                                              \
    cudaError_t e_ = cudaGetLastError();                                            \
    if (e_ != cudaSuccess) {                                                        \
      pf5d::set_error("%s:%d launch: %s", __FILE__, __LINE__, cudaGetErrorString(e_)); \
      return PF5D_ERR_CUDA;                                                         \
    }                                                                               \
  } while (0)

#define PF5D_REQUIRE(cond, code, ...)                                               \
  do {                                                                              \
    if (!(cond)) {                                                                  \
      pf5d::set_error(__VA_ARGS__);                                                 \
      return (code);                                                                \
    }                                                                               \
  } while (0)
