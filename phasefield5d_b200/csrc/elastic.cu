// elastic.cu -- rank-1 Khachaturyan elastic term around one cuFFT pair
// (phasefield5d/solver/elastic.py:147-263, scipy path 242-263):
//   s(x)  = sum_s (X[x,s] - X0[s]) * l[s]            (k_misfit, elastic.py:21-29)
//   S(k)  = rfftn(s) * B(k)                          (cuFFT D2Z + k_bmul)
//   s'(x) = irfftn(S)                                (cuFFT Z2D; 1/N folded into B)
//   mu   += s'(x) * l                                (k_expand_add)
// Compiled with -fmad=false.
#include <cmath>
#include <vector>

#include "pf5d_device.cuh"
#include "pf5d_fft.h"
#include "pf5d_stockham.cuh"

namespace pf5d {

#define PF5D_CUFFT(call)                                                           \
  do {                                                                             \
    cufftResult r_ = (call);                                                       \
    if (r_ != CUFFT_SUCCESS) {                                                     \
      set_error("%s:%d %s: cufft error %d", __FILE__, __LINE__, #call, (int)r_);   \
      return PF5D_ERR_CUFFT;                                                       \
    }                                                                              \
  } while (0)

pf5d_status fft_create(int dim, const int64_t *shape, FFTPair *p) {
  PF5D_REQUIRE(dim >= 1 && dim <= 3, PF5D_ERR_DIM,
               "make_elastic_updater not implemented for spatial_dim=%d", dim);
  long long n[3];
  int64_t npts = 1;
  for (int d = 0; d < dim; ++d) {
    PF5D_REQUIRE(shape[d] > 0, PF5D_ERR_ARG, "bad shape");
    n[d] = shape[d];
    npts *= shape[d];
  }
  const int64_t nk = npts / shape[dim - 1] * (shape[dim - 1] / 2 + 1);
  size_t ws = 0;
  PF5D_CUFFT(cufftCreate(&p->fwd));
  PF5D_CUFFT(cufftMakePlanMany64(p->fwd, dim, n, nullptr, 1, 0, nullptr, 1, 0, CUFFT_D2Z, 1, &ws));
  PF5D_CUFFT(cufftCreate(&p->inv));
  PF5D_CUFFT(cufftMakePlanMany64(p->inv, dim, n, nullptr, 1, 0, nullptr, 1, 0, CUFFT_Z2D, 1, &ws));
  p->npts = npts;
  p->nk = nk;
  p->ready = true;
  return PF5D_OK;
}

void fft_destroy(FFTPair *p) {
  if (p->ready) {
    cufftDestroy(p->fwd);
    cufftDestroy(p->inv);
  }
  p->ready = false;
}

pf5d_status fft_forward(FFTPair *p, double *s, cufftDoubleComplex *k, cudaStream_t stream) {
  PF5D_CUFFT(cufftSetStream(p->fwd, stream));
  PF5D_CUFFT(cufftExecD2Z(p->fwd, s, k));
  return PF5D_OK;
}

pf5d_status fft_inverse(FFTPair *p, cufftDoubleComplex *k, double *s, cudaStream_t stream) {
  PF5D_CUFFT(cufftSetStream(p->inv, stream));
  PF5D_CUFFT(cufftExecZ2D(p->inv, k, s));
  return PF5D_OK;
}

// ------------------------------------------------------------------------
// 2D column pass: for a group of kColGroup spectrum columns (axis-1 indices
// of the row transforms' output), the length-N0 transform along axis 0, the
// B(k)/N multiply and the inverse transform, in shared memory.  Transforms:
// mixed-radix Stockham autosort (radix-8 stages, then one radix-4 or radix-2
// stage; natural order after every stage), forward exp(-2 pi i jk/N0),
// inverse exp(+2 pi i jk/N0), both unnormalised like cuFFT's (the 1/N is
// in B).
// ------------------------------------------------------------------------
constexpr int kColGroup = 1;

template <typename C, int N0>
__global__ void __launch_bounds__(kColThreads)
    k_colpass(C *__restrict__ k, const typename CT<C>::R *__restrict__ bk, int nk1,
              const C *__restrict__ tw, const unsigned *halt) {
  extern __shared__ __align__(16) unsigned char craw[];
  C *cbuf = reinterpret_cast<C *>(craw);             // [2][kColGroup][N0]
  if (halt && *halt) return;
  const int tid = threadIdx.x, c0 = blockIdx.x * kColGroup;
  C *a = cbuf, *b = cbuf + kColGroup * N0;
  C *kk = k;
  for (int e = tid; e < kColGroup * N0; e += kColThreads) {
    const int r = e / kColGroup, cc = e - r * kColGroup, c = c0 + cc;
    a[cc * N0 + r] = c < nk1 ? kk[(int64_t)r * nk1 + c] : cmk<C>(0, 0);
  }
  __syncthreads();
  C *f = stockham<C, N0, false>(a, b, tw, tid);
  C *g = f == a ? b : a;
  for (int e = tid; e < kColGroup * N0; e += kColThreads) {
    const int cc = e / N0, r = e - cc * N0, c = c0 + cc;
    const typename CT<C>::R m = c < nk1 ? bk[(int64_t)r * nk1 + c] : 0;
    C v = f[e];
    v.x = v.x * m;
    v.y = v.y * m;
    f[e] = v;
  }
  __syncthreads();
  f = stockham<C, N0, true>(f, g, tw, tid);
  for (int e = tid; e < kColGroup * N0; e += kColThreads) {
    const int r = e / kColGroup, cc = e - r * kColGroup, c = c0 + cc;
    if (c < nk1) kk[(int64_t)r * nk1 + c] = f[cc * N0 + r];
  }
}

template <typename C>
static pf5d_status colpass_dispatch(const ColPass2D *c, C *k, const typename CT<C>::R *bk,
                                    const C *tw, const unsigned *halt, cudaStream_t stream);

pf5d_status colpass_create(const int64_t *shape, ColPass2D *c, bool fp32) {
  const int64_t n0 = shape[0], n1 = shape[1];
  PF5D_REQUIRE(n0 >= 8 && n0 <= 1024 && (n0 & (n0 - 1)) == 0 && n1 >= 2, PF5D_ERR_ARG,
               "column pass needs a power-of-two axis 0 in [8, 1024]");
  c->n0 = (int)n0;
  c->nk1 = (int)(n1 / 2 + 1);
  c->fp32 = fp32;
  long long n[1] = {(long long)n1};
  size_t ws = 0;
  PF5D_CUFFT(cufftCreate(&c->rfwd));
  PF5D_CUFFT(cufftMakePlanMany64(c->rfwd, 1, n, nullptr, 1, 0, nullptr, 1, 0,
                                 fp32 ? CUFFT_R2C : CUFFT_D2Z, n0, &ws));
  PF5D_CUFFT(cufftCreate(&c->rinv));
  PF5D_CUFFT(cufftMakePlanMany64(c->rinv, 1, n, nullptr, 1, 0, nullptr, 1, 0,
                                 fp32 ? CUFFT_C2R : CUFFT_Z2D, n0, &ws));
  c->ready = true;
  // exp(-2 pi i m / n0) in FP64, rounded once for the FP32 form
  std::vector<double2> tw(n0);
  std::vector<float2> tw32(n0);
  const double pi = 3.14159265358979323846;
  for (int64_t m = 0; m < n0; ++m) {
    const double ang = 2.0 * pi * (double)m / (double)n0;
    tw[m] = make_double2(std::cos(ang), -std::sin(ang));
    tw32[m] = make_float2((float)tw[m].x, (float)tw[m].y);
  }
  if (fp32) {
    PF5D_CUDA(cudaMalloc(&c->tw32, tw32.size() * sizeof(float2)));
    PF5D_CUDA(cudaMemcpy(c->tw32, tw32.data(), tw32.size() * sizeof(float2), cudaMemcpyHostToDevice));
    return colpass_dispatch<float2>(c, nullptr, nullptr, nullptr, nullptr, nullptr);
  }
  PF5D_CUDA(cudaMalloc(&c->tw, tw.size() * sizeof(double2)));
  PF5D_CUDA(cudaMemcpy(c->tw, tw.data(), tw.size() * sizeof(double2), cudaMemcpyHostToDevice));
  return colpass_dispatch<double2>(c, nullptr, nullptr, nullptr, nullptr, nullptr);
}

void colpass_destroy(ColPass2D *c) {
  if (c->ready) {
    cufftDestroy(c->rfwd);
    cufftDestroy(c->rinv);
  }
  cudaFree(c->tw);
  cudaFree(c->tw32);
  c->tw = nullptr;
  c->tw32 = nullptr;
  c->ready = false;
}

pf5d_status colpass_rows_forward(ColPass2D *c, double *s, cufftDoubleComplex *k,
                                 cudaStream_t stream) {
  PF5D_CUFFT(cufftSetStream(c->rfwd, stream));
  PF5D_CUFFT(cufftExecD2Z(c->rfwd, s, k));
  return PF5D_OK;
}

pf5d_status colpass_rows_inverse(ColPass2D *c, cufftDoubleComplex *k, double *s,
                                 cudaStream_t stream) {
  PF5D_CUFFT(cufftSetStream(c->rinv, stream));
  PF5D_CUFFT(cufftExecZ2D(c->rinv, k, s));
  return PF5D_OK;
}

template <typename C, int N0>
static pf5d_status launch_colpass(const ColPass2D *c, C *k, const typename CT<C>::R *bk,
                                  const C *tw, const unsigned *halt, cudaStream_t stream) {
  const int smem = 2 * N0 * (int)sizeof(C);
  if (!k) {                          // set-up call from colpass_create
    PF5D_CUDA(cudaFuncSetAttribute(k_colpass<C, N0>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   smem));
    return PF5D_OK;
  }
  k_colpass<C, N0><<<(unsigned)c->nk1, kColThreads, smem, stream>>>(k, bk, c->nk1, tw, halt);
  PF5D_LAUNCHED();
  return PF5D_OK;
}

template <typename C>
static pf5d_status colpass_dispatch(const ColPass2D *c, C *k, const typename CT<C>::R *bk,
                                    const C *tw, const unsigned *halt, cudaStream_t stream) {
  switch (c->n0) {
    case 8: return launch_colpass<C, 8>(c, k, bk, tw, halt, stream);
    case 16: return launch_colpass<C, 16>(c, k, bk, tw, halt, stream);
    case 32: return launch_colpass<C, 32>(c, k, bk, tw, halt, stream);
    case 64: return launch_colpass<C, 64>(c, k, bk, tw, halt, stream);
    case 128: return launch_colpass<C, 128>(c, k, bk, tw, halt, stream);
    case 256: return launch_colpass<C, 256>(c, k, bk, tw, halt, stream);
    case 512: return launch_colpass<C, 512>(c, k, bk, tw, halt, stream);
    case 1024: return launch_colpass<C, 1024>(c, k, bk, tw, halt, stream);
    default: set_error("column pass: unsupported n0 %d", c->n0); return PF5D_ERR_ARG;
  }
}

pf5d_status colpass_columns(ColPass2D *c, cufftDoubleComplex *k, const double *bk,
                            const unsigned *halt, cudaStream_t stream) {
  return colpass_dispatch<double2>(c, reinterpret_cast<double2 *>(k), bk, c->tw, halt, stream);
}

pf5d_status colpass_columns32(ColPass2D *c, cufftComplex *k, const float *bk,
                              const unsigned *halt, cudaStream_t stream) {
  return colpass_dispatch<float2>(c, reinterpret_cast<float2 *>(k), bk, c->tw32, halt, stream);
}

pf5d_status colpass_rows_forward32(ColPass2D *c, float *s, cufftComplex *k, cudaStream_t stream) {
  PF5D_CUFFT(cufftSetStream(c->rfwd, stream));
  PF5D_CUFFT(cufftExecR2C(c->rfwd, s, k));
  return PF5D_OK;
}

pf5d_status colpass_rows_inverse32(ColPass2D *c, cufftComplex *k, float *s, cudaStream_t stream) {
  PF5D_CUFFT(cufftSetStream(c->rinv, stream));
  PF5D_CUFFT(cufftExecC2R(c->rinv, k, s));
  return PF5D_OK;
}

__global__ void k_misfit(const double *__restrict__ X, int64_t npts, Vec4 x0, Vec4 l,
                         double *__restrict__ s, const unsigned *halt) {
  if (halt && *halt) return;
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < npts;
       p += (int64_t)gridDim.x * blockDim.x) {
    const double2 a = reinterpret_cast<const double2 *>(X + 4 * p)[0];
    const double2 b = reinterpret_cast<const double2 *>(X + 4 * p)[1];
    double acc = 0.0;
    acc = acc + (a.x - x0.v[0]) * l.v[0];
    acc = acc + (a.y - x0.v[1]) * l.v[1];
    acc = acc + (b.x - x0.v[2]) * l.v[2];
    acc = acc + (b.y - x0.v[3]) * l.v[3];
    s[p] = acc;
  }
}

// numpy's complex *= real multiplies both parts by the real factor.
__global__ void k_bmul(cufftDoubleComplex *__restrict__ k, const double *__restrict__ bk,
                       int64_t nk, const unsigned *halt) {
  if (halt && *halt) return;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nk;
       i += (int64_t)gridDim.x * blockDim.x) {
    const double b = bk[i];
    cufftDoubleComplex v = k[i];
    v.x = v.x * b;
    v.y = v.y * b;
    k[i] = v;
  }
}

__global__ void k_expand_add(double *mu, int64_t mus, const double *__restrict__ s, Vec4 l,
                             int64_t npts) {
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < npts;
       p += (int64_t)gridDim.x * blockDim.x) {
    const double sv = s[p];
#pragma unroll
    for (int c = 0; c < 4; ++c) mu[p * mus + c] = mu[p * mus + c] + sv * l.v[c];
  }
}

pf5d_status launch_misfit(const double *X, int64_t npts, Vec4 x0, Vec4 l, double *s,
                          const unsigned *halt, cudaStream_t stream) {
  k_misfit<<<grid_for(npts, 256), 256, 0, stream>>>(X, npts, x0, l, s, halt);
  PF5D_LAUNCHED();
  return PF5D_OK;
}

pf5d_status launch_bmul(cufftDoubleComplex *k, const double *bk, int64_t nk, const unsigned *halt,
                        cudaStream_t stream) {
  k_bmul<<<grid_for(nk, 256), 256, 0, stream>>>(k, bk, nk, halt);
  PF5D_LAUNCHED();
  return PF5D_OK;
}

pf5d_status launch_expand_add(double *mu, int64_t mu_stride, const double *s, Vec4 l,
                              int64_t npts, cudaStream_t stream) {
  k_expand_add<<<grid_for(npts, 256), 256, 0, stream>>>(mu, mu_stride, s, l, npts);
  PF5D_LAUNCHED();
  return PF5D_OK;
}

pf5d_status upload_bk_scaled(const double *bk_host, int64_t nk, int64_t npts, double **bk_dev) {
  std::vector<double> h(nk);
  const double inv_n = 1.0 / (double)npts;
  for (int64_t i = 0; i < nk; ++i) h[i] = bk_host[i] * inv_n;
  PF5D_CUDA(cudaMalloc(bk_dev, nk * sizeof(double)));
  PF5D_CUDA(cudaMemcpy(*bk_dev, h.data(), nk * sizeof(double), cudaMemcpyHostToDevice));
  return PF5D_OK;
}

}  // namespace pf5d

using namespace pf5d;

struct pf5d_elastic {
  int dim = 0;
  Vec4 x0{}, l{};
  FFTPair fft;
  double *bk = nullptr;
  double *s = nullptr;
  cufftDoubleComplex *k = nullptr;
};

extern "C" {

pf5d_status pf5d_elastic_create(int32_t dim, const int64_t *shape, const double *x0,
                                const double *lvec, const double *bk, pf5d_elastic **out) {
  PF5D_REQUIRE(out && shape && x0 && lvec && bk, PF5D_ERR_ARG, "null argument");
  auto *h = new pf5d_elastic();
  h->dim = dim;
  for (int c = 0; c < 4; ++c) {
    h->x0.v[c] = x0[c];
    h->l.v[c] = lvec[c];
  }
  pf5d_status st = fft_create(dim, shape, &h->fft);
  if (st == PF5D_OK) st = upload_bk_scaled(bk, h->fft.nk, h->fft.npts, &h->bk);
  if (st == PF5D_OK && cudaMalloc(&h->s, h->fft.npts * sizeof(double)) != cudaSuccess)
    st = PF5D_ERR_CUDA;
  if (st == PF5D_OK && cudaMalloc(&h->k, h->fft.nk * sizeof(cufftDoubleComplex)) != cudaSuccess)
    st = PF5D_ERR_CUDA;
  if (st != PF5D_OK) {
    pf5d_elastic_destroy(h);
    return st;
  }
  *out = h;
  return PF5D_OK;
}

pf5d_status pf5d_elastic_apply(pf5d_elastic *h, double *mu, int64_t mu_stride, const double *X,
                               void *stream) {
  PF5D_REQUIRE(h && mu && X && mu_stride >= 4, PF5D_ERR_ARG, "bad arguments");
  PF5D_REQUIRE(((uintptr_t)X & 15) == 0, PF5D_ERR_ARG, "X must be 16-byte aligned");
  cudaStream_t s = as_stream(stream);
  pf5d_status st;
  if ((st = launch_misfit(X, h->fft.npts, h->x0, h->l, h->s, nullptr, s)) != PF5D_OK) return st;
  if ((st = fft_forward(&h->fft, h->s, h->k, s)) != PF5D_OK) return st;
  if ((st = launch_bmul(h->k, h->bk, h->fft.nk, nullptr, s)) != PF5D_OK) return st;
  if ((st = fft_inverse(&h->fft, h->k, h->s, s)) != PF5D_OK) return st;
  return launch_expand_add(mu, mu_stride, h->s, h->l, h->fft.npts, s);
}

pf5d_status pf5d_elastic_destroy(pf5d_elastic *h) {
  if (!h) return PF5D_OK;
  fft_destroy(&h->fft);
  cudaFree(h->bk);
  cudaFree(h->s);
  cudaFree(h->k);
  delete h;
  return PF5D_OK;
}

}  // extern "C"
