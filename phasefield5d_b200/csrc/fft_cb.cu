// fft_cb.cu -- inverse-transform plans with the B(k) multiply fused in as an
// LTO load callback (bk_callbacks.cu, embedded as a fatbin).  When the
// callback cannot be attached or linked, the plan is made without it and the
// caller keeps its stand-alone multiply kernel.
#include <cufftXt.h>

#include "pf5d_fft.h"
#include "bk_callbacks_fatbin.h"   // generated: kBkCallbacksFatbin

namespace pf5d {

namespace {
struct BkInfo {
  const void *bk;
  unsigned long long nk;
};
}  // namespace

cufftResult make_inverse_plan(cufftHandle *plan, int rank, long long *n, long long idist,
                              long long odist, cufftType type, long long batch,
                              const void *bk_dev, long long nk, void **info_dev, bool *fused) {
  *fused = false;
  *info_dev = nullptr;
  size_t ws = 0;
  cufftResult r = cufftCreate(plan);
  if (r != CUFFT_SUCCESS) return r;
  if (bk_dev) {
    BkInfo h{bk_dev, (unsigned long long)nk};
    const bool fp64 = type == CUFFT_Z2D;
    const char *name = fp64 ? "pf5d_bk_load_z" : (batch > 1 ? "pf5d_bk_load_c_batch" : "pf5d_bk_load_c");
    if (cudaMalloc(info_dev, sizeof(BkInfo)) == cudaSuccess &&
        cudaMemcpy(*info_dev, &h, sizeof(BkInfo), cudaMemcpyHostToDevice) == cudaSuccess &&
        cufftXtSetJITCallback(*plan, name, kBkCallbacksFatbin, sizeof(kBkCallbacksFatbin),
                              fp64 ? CUFFT_CB_LD_COMPLEX_DOUBLE : CUFFT_CB_LD_COMPLEX,
                              info_dev) == CUFFT_SUCCESS) {
      r = cufftMakePlanMany64(*plan, rank, n, nullptr, 1, idist, nullptr, 1, odist, type, batch, &ws);
      if (r == CUFFT_SUCCESS) {
        *fused = true;
        return r;
      }
    }
    // no callback: a plain plan, the caller multiplies with its own kernel
    cufftDestroy(*plan);
    if (*info_dev) cudaFree(*info_dev);
    *info_dev = nullptr;
    cudaGetLastError();
    r = cufftCreate(plan);
    if (r != CUFFT_SUCCESS) return r;
  }
  return cufftMakePlanMany64(*plan, rank, n, nullptr, 1, idist, nullptr, 1, odist, type, batch, &ws);
}

}  // namespace pf5d
