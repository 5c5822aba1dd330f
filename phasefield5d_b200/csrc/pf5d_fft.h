// pf5d_fft.h -- the rank-1 elastic operator's cuFFT plan pair and the
// hand-written kernels around it (misfit contraction, B(k) multiply, rank-1
// expansion), shared by the drop-in elastic handle and the step loop.
#pragma once

#include <cstdint>
#include <cufft.h>

#include "pf5d_host.h"

namespace pf5d {

// D2Z / Z2D plans over a 1D/2D/3D real field of `shape` (C order); the
// half-spectrum has shape[:-1] x (shape[-1]/2 + 1) complex values, the layout
// of numpy's rfftn.
struct FFTPair {
  cufftHandle fwd = 0, inv = 0;
  int64_t npts = 0, nk = 0;
  bool ready = false;
};

pf5d_status fft_create(int dim, const int64_t *shape, FFTPair *p);
void fft_destroy(FFTPair *p);
// s (real, npts) -> k (complex, nk); k -> s.  Both on `stream`.
pf5d_status fft_forward(FFTPair *p, double *s, cufftDoubleComplex *k, cudaStream_t stream);
pf5d_status fft_inverse(FFTPair *p, cufftDoubleComplex *k, double *s, cudaStream_t stream);

// 2D elastic term in three passes instead of cuFFT's four plus the multiply:
// row D2Z over axis 1 (cuFFT, batched over the n0 rows), then ONE kernel per
// group of spectrum columns that runs the length-n0 transform along axis 0,
// multiplies by B(k)/N and runs the inverse transform back (k_colpass), then
// row Z2D.  Used when n0 is a power of two in [8, 1024].
struct ColPass2D {
  cufftHandle rfwd = 0, rinv = 0;     // batched row transforms
  int n0 = 0, nk1 = 0;                // rows, spectrum columns (n1/2 + 1)
  double2 *tw = nullptr;              // exp(-2 pi i m / n0), m < n0 (FP64 form)
  float2 *tw32 = nullptr;             // the same rounded to FP32 (FP32c form)
  bool fp32 = false;                  // FP32c: R2C / C2R rows, float2 spectrum
  bool ready = false;
};

pf5d_status colpass_create(const int64_t *shape, ColPass2D *c, bool fp32);
void colpass_destroy(ColPass2D *c);
// s -> s' in place through k (scratch spectrum), bk = B(k)/N on the half grid.
pf5d_status colpass_rows_forward(ColPass2D *c, double *s, cufftDoubleComplex *k,
                                 cudaStream_t stream);
pf5d_status colpass_columns(ColPass2D *c, cufftDoubleComplex *k, const double *bk,
                            const unsigned *halt, cudaStream_t stream);
pf5d_status colpass_rows_inverse(ColPass2D *c, cufftDoubleComplex *k, double *s,
                                 cudaStream_t stream);
// The FP32c form's passes (float field, cufftComplex spectrum, B(k)/N in FP32).
pf5d_status colpass_rows_forward32(ColPass2D *c, float *s, cufftComplex *k, cudaStream_t stream);
pf5d_status colpass_columns32(ColPass2D *c, cufftComplex *k, const float *bk,
                              const unsigned *halt, cudaStream_t stream);
pf5d_status colpass_rows_inverse32(ColPass2D *c, cufftComplex *k, float *s, cudaStream_t stream);

struct Vec4 {
  double v[4];
};

// Device-side step-state halt word the step-loop kernels honour (nullptr: none).
pf5d_status launch_misfit(const double *X, int64_t npts, Vec4 x0, Vec4 l, double *s,
                          const unsigned *halt, cudaStream_t stream);
pf5d_status launch_bmul(cufftDoubleComplex *k, const double *bk, int64_t nk, const unsigned *halt,
                        cudaStream_t stream);
pf5d_status launch_expand_add(double *mu, int64_t mu_stride, const double *s, Vec4 l,
                              int64_t npts, cudaStream_t stream);

// Host B(k) scaled by 1/N (the inverse transform's normalisation) into a new
// device buffer.
pf5d_status upload_bk_scaled(const double *bk_host, int64_t nk, int64_t npts, double **bk_dev);

}  // namespace pf5d
