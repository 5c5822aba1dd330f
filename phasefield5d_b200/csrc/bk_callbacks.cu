// bk_callbacks.cu -- the elastic operator's B(k) multiply as cuFFT load
// callbacks of the inverse (half-spectrum -> real) transforms.  Built only as
// LTO IR (nvcc -rdc -dlto, code=lto_100a) and embedded in the library; cuFFT
// links it into its own kernels when the inverse plan is made, so the
// multiply costs no launch and no extra pass over the spectrum.  Each
// element is multiplied exactly as the stand-alone kernels do it (both
// parts by the real factor B(k)/N), so the values match them bit for bit.
#include <cufftXt.h>

struct Pf5dBkInfo {
  const void *bk;            // B(k)/N on the half-spectrum (double or float)
  unsigned long long nk;     // half-spectrum length of one transform
};

extern "C" __device__ cufftDoubleComplex pf5d_bk_load_z(void *in, unsigned long long off,
                                                        void *info, void *) {
  const Pf5dBkInfo *p = static_cast<const Pf5dBkInfo *>(info);
  cufftDoubleComplex v = static_cast<const cufftDoubleComplex *>(in)[off];
  const double b = static_cast<const double *>(p->bk)[off];
  v.x = v.x * b;
  v.y = v.y * b;
  return v;
}

extern "C" __device__ cufftComplex pf5d_bk_load_c(void *in, unsigned long long off, void *info,
                                                  void *) {
  const Pf5dBkInfo *p = static_cast<const Pf5dBkInfo *>(info);
  cufftComplex v = static_cast<const cufftComplex *>(in)[off];
  const float b = static_cast<const float *>(p->bk)[off];
  v.x *= b;
  v.y *= b;
  return v;
}

// A batch of same-shape transforms shares one B(k)/N.
extern "C" __device__ cufftComplex pf5d_bk_load_c_batch(void *in, unsigned long long off,
                                                        void *info, void *) {
  const Pf5dBkInfo *p = static_cast<const Pf5dBkInfo *>(info);
  cufftComplex v = static_cast<const cufftComplex *>(in)[off];
  const float b = static_cast<const float *>(p->bk)[off % p->nk];
  v.x *= b;
  v.y *= b;
  return v;
}
