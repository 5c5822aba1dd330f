// ops.cu -- one device kernel per reference hot-path function, behind the
// C ABI of include/pf5d.h.  These are the drop-in forms of the reference's
// separate passes (interpolator_nb, calculate_laplacian, the fused divergence,
// abs_max, clamp_simplex, the update, out_of_bounds); the fused step loop in
// stepper.cu reuses the same device routines.
//
// Compiled with -fmad=false: FP64 results equal the reference's Numba kernels
// bit for bit.
#include <cmath>
#include <cstring>
#include <mutex>
#include <vector>

#include "pf5d_device.cuh"
#include "pf5d_host.h"

namespace pf5d {

static thread_local std::string g_last_error;

void set_error(const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
}

int sm_count() {
  static int cached[64] = {0};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= 64) dev = 0;
  if (cached[dev] == 0) {
    int n = 0;
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    cached[dev] = n > 0 ? n : 148;
  }
  return cached[dev];
}

// ------------------------------------------------------------------ interp
__global__ void k_interp4d(const double *__restrict__ comp, int64_t npts, Table T,
                           double *__restrict__ out, int64_t out_stride, uint8_t *mask,
                           unsigned *flags) {
  unsigned f = 0;
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < npts;
       r += (int64_t)gridDim.x * blockDim.x) {
    double x[S];
    const double2 a = reinterpret_cast<const double2 *>(comp + 4 * r)[0];
    const double2 b = reinterpret_cast<const double2 *>(comp + 4 * r)[1];
    x[0] = a.x; x[1] = a.y; x[2] = b.x; x[3] = b.y;
    double v[NP];
    const bool lin = interp_point(T, x, v, &f);
    if (mask) mask[r] = lin ? 1 : 0;
    double *o = out + r * out_stride;
#pragma unroll
    for (int p = 0; p < NP; ++p) o[p] = v[p];
  }
  if (flags && f) atomicOr(flags, f);
}

// --------------------------------------------------------------- laplacian
// operators.py:32-76; neighbour order +axis0, -axis0, +axis1, -axis1, +axis2, -axis2.
__global__ void k_laplacian(int dim, int64_t n0, int64_t n1, int64_t n2, int nc,
                            const double *__restrict__ c, double inv_dx2,
                            double *__restrict__ out) {
  const int64_t npts = n0 * n1 * n2;
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < npts;
       p += (int64_t)gridDim.x * blockDim.x) {
    const int64_t k = p % n2, j = (p / n2) % n1, i = p / (n2 * n1);
    if (dim == 1) {
      const int64_t ip = wrap_p(i, n0), im = wrap_m(i, n0);
      for (int s = 0; s < nc; ++s)
        out[p * nc + s] = (c[ip * nc + s] + c[im * nc + s] - 2.0 * c[p * nc + s]) * inv_dx2;
    } else if (dim == 2) {
      const int64_t ip = wrap_p(i, n0) * n1 + j, im = wrap_m(i, n0) * n1 + j;
      const int64_t jp = i * n1 + wrap_p(j, n1), jm = i * n1 + wrap_m(j, n1);
      for (int s = 0; s < nc; ++s)
        out[p * nc + s] = (c[ip * nc + s] + c[im * nc + s] + c[jp * nc + s] + c[jm * nc + s] -
                           4.0 * c[p * nc + s]) * inv_dx2;
    } else {
      const int64_t ip = (wrap_p(i, n0) * n1 + j) * n2 + k, im = (wrap_m(i, n0) * n1 + j) * n2 + k;
      const int64_t jp = (i * n1 + wrap_p(j, n1)) * n2 + k, jm = (i * n1 + wrap_m(j, n1)) * n2 + k;
      const int64_t kp = (i * n1 + j) * n2 + wrap_p(k, n2), km = (i * n1 + j) * n2 + wrap_m(k, n2);
      for (int s = 0; s < nc; ++s)
        out[p * nc + s] = (c[ip * nc + s] + c[im * nc + s] + c[jp * nc + s] + c[jm * nc + s] +
                           c[kp * nc + s] + c[km * nc + s] - 6.0 * c[p * nc + s]) * inv_dx2;
    }
  }
}

struct Kappa {
  double k[8];
};

__global__ void k_kappa_subtract(double *mu, int64_t mu_stride, double *lap, Kappa kap,
                                 int64_t npts, int nc) {
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < npts;
       p += (int64_t)gridDim.x * blockDim.x)
    for (int s = 0; s < nc; ++s) {
      const double l = lap[p * nc + s] * kap.k[s];
      lap[p * nc + s] = l;
      mu[p * mu_stride + s] = mu[p * mu_stride + s] - l;
    }
}

// ------------------------------------------------------------- divergence
// fluxes.py:296-395: per point, both faces per axis (gradients inline), then
// (f0p - f0m + f1p - f1m + f2p - f2m) * inv_dx left to right.
__device__ __forceinline__ void load4(const double *p, double v[S]) {
#pragma unroll
  for (int s = 0; s < S; ++s) v[s] = p[s];
}
__device__ __forceinline__ void load5(const double *p, double v[NM]) {
#pragma unroll
  for (int s = 0; s < NM; ++s) v[s] = p[s];
}

__global__ void k_divergence(int dim, int64_t n0, int64_t n1, int64_t n2,
                             const double *__restrict__ X, const double *__restrict__ M,
                             int64_t ms, const double *__restrict__ mu, int64_t mus,
                             double inv_dx, double *__restrict__ out) {
  const int64_t npts = n0 * n1 * n2;
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < npts;
       p += (int64_t)gridDim.x * blockDim.x) {
    const int64_t k = p % n2, j = (p / n2) % n1, i = p / (n2 * n1);
    int64_t nb[6];
    nb[0] = (wrap_p(i, n0) * n1 + j) * n2 + k;
    nb[1] = (wrap_m(i, n0) * n1 + j) * n2 + k;
    nb[2] = (i * n1 + wrap_p(j, n1)) * n2 + k;
    nb[3] = (i * n1 + wrap_m(j, n1)) * n2 + k;
    nb[4] = (i * n1 + j) * n2 + wrap_p(k, n2);
    nb[5] = (i * n1 + j) * n2 + wrap_m(k, n2);
    double Xc[S], Mc[NM], muc[S];
    load4(X + p * S, Xc);
    load5(M + p * ms, Mc);
    load4(mu + p * mus, muc);
    double acc[S];
    for (int f = 0; f < 2 * dim; ++f) {
      const int64_t q = nb[f];
      double Xn[S], Mn[NM], mun[S], g[S], J[S];
      load4(X + q * S, Xn);
      load5(M + q * ms, Mn);
      load4(mu + q * mus, mun);
#pragma unroll
      for (int s = 0; s < S; ++s) g[s] = (f & 1) ? (muc[s] - mun[s]) * inv_dx : (mun[s] - muc[s]) * inv_dx;
      face_flux(Xc, Mc, Xn, Mn, g, J);
#pragma unroll
      for (int s = 0; s < S; ++s) {
        if (f == 0) acc[s] = J[s];
        else if (f & 1) acc[s] = acc[s] - J[s];
        else acc[s] = acc[s] + J[s];
      }
    }
#pragma unroll
    for (int s = 0; s < S; ++s) out[p * S + s] = acc[s] * inv_dx;
  }
}

// ---------------------------------------------- save-step gradients/fluxes
__global__ void k_gradients_pm(int dim, int64_t n0, int64_t n1, int64_t n2, int nc,
                               const double *__restrict__ c, int64_t cs, double inv_dx,
                               double *__restrict__ gp, double *__restrict__ gm) {
  const int64_t npts = n0 * n1 * n2;
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < npts;
       p += (int64_t)gridDim.x * blockDim.x) {
    const int64_t k = p % n2, j = (p / n2) % n1, i = p / (n2 * n1);
    int64_t pp[3], pm[3];
    pp[0] = (wrap_p(i, n0) * n1 + j) * n2 + k;
    pm[0] = (wrap_m(i, n0) * n1 + j) * n2 + k;
    pp[1] = (i * n1 + wrap_p(j, n1)) * n2 + k;
    pm[1] = (i * n1 + wrap_m(j, n1)) * n2 + k;
    pp[2] = (i * n1 + j) * n2 + wrap_p(k, n2);
    pm[2] = (i * n1 + j) * n2 + wrap_m(k, n2);
    for (int d = 0; d < dim; ++d)
      for (int s = 0; s < nc; ++s) {
        const double center = c[p * cs + s];
        gp[(d * npts + p) * nc + s] = (c[pp[d] * cs + s] - center) * inv_dx;
        gm[(d * npts + p) * nc + s] = (center - c[pm[d] * cs + s]) * inv_dx;
      }
  }
}

__global__ void k_fluxes_pm(int dim, int64_t n0, int64_t n1, int64_t n2,
                            const double *__restrict__ X, const double *__restrict__ M, int64_t ms,
                            const double *__restrict__ gp, const double *__restrict__ gm,
                            double *__restrict__ fp, double *__restrict__ fm) {
  const int64_t npts = n0 * n1 * n2;
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < npts;
       p += (int64_t)gridDim.x * blockDim.x) {
    const int64_t k = p % n2, j = (p / n2) % n1, i = p / (n2 * n1);
    int64_t pp[3], pm[3];
    pp[0] = (wrap_p(i, n0) * n1 + j) * n2 + k;
    pm[0] = (wrap_m(i, n0) * n1 + j) * n2 + k;
    pp[1] = (i * n1 + wrap_p(j, n1)) * n2 + k;
    pm[1] = (i * n1 + wrap_m(j, n1)) * n2 + k;
    pp[2] = (i * n1 + j) * n2 + wrap_p(k, n2);
    pm[2] = (i * n1 + j) * n2 + wrap_m(k, n2);
    double Xc[S], Mc[NM];
    load4(X + p * S, Xc);
    load5(M + p * ms, Mc);
    for (int d = 0; d < dim; ++d) {
      const int64_t o = (d * npts + p) * S;
      double Xn[S], Mn[NM], g[S], J[S];
      load4(X + pp[d] * S, Xn);
      load5(M + pp[d] * ms, Mn);
      load4(gp + o, g);
      face_flux(Xc, Mc, Xn, Mn, g, J);
#pragma unroll
      for (int s = 0; s < S; ++s) fp[o + s] = J[s];
      load4(X + pm[d] * S, Xn);
      load5(M + pm[d] * ms, Mn);
      load4(gm + o, g);
      face_flux(Xc, Mc, Xn, Mn, g, J);
#pragma unroll
      for (int s = 0; s < S; ++s) fm[o + s] = J[s];
    }
  }
}

// ------------------------------------------------------------- reductions
constexpr int kAbsMaxBlocks = 1024;
constexpr int kAbsMaxThreads = 256;

// Pass 1: per-block max |a| (NaN ignored, like `if v > m: m = v`).
__global__ void k_absmax_partial(const double *__restrict__ a, int64_t n,
                                 double *__restrict__ partial) {
  __shared__ double red[kAbsMaxThreads / 32];
  double m = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const double v = fabs(a[i]);
    if (v > m) m = v;
  }
  m = block_max<kAbsMaxThreads>(m, red);
  if (threadIdx.x == 0) partial[blockIdx.x] = m;
}

// Pass 2: one block folds the partials into *result.
__global__ void k_absmax_final(const double *__restrict__ partial, int nparts, double *result) {
  __shared__ double red[kAbsMaxThreads / 32];
  double m = 0.0;
  for (int i = threadIdx.x; i < nparts; i += blockDim.x) m = fmax(m, partial[i]);
  m = block_max<kAbsMaxThreads>(m, red);
  if (threadIdx.x == 0) *result = m;
}

// Per-device workspace for the block partials of abs_max (allocated once).
static std::mutex g_ws_mutex;
static double *g_absmax_ws[64] = {nullptr};

static pf5d_status absmax_workspace(double **out) {
  int dev = 0;
  PF5D_CUDA(cudaGetDevice(&dev));
  PF5D_REQUIRE(dev >= 0 && dev < 64, PF5D_ERR_ARG, "device ordinal %d out of range", dev);
  std::lock_guard<std::mutex> lock(g_ws_mutex);
  if (!g_absmax_ws[dev]) PF5D_CUDA(cudaMalloc(&g_absmax_ws[dev], kAbsMaxBlocks * sizeof(double)));
  *out = g_absmax_ws[dev];
  return PF5D_OK;
}

__global__ void k_clamp(double *X, int64_t npts, int nc) {
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < npts;
       p += (int64_t)gridDim.x * blockDim.x) {
    double total = 0.0;
    for (int s = 0; s < nc; ++s) total = total + X[p * nc + s];
    if (total > 1.0) {
      const double inv = 1.0 / total;
      for (int s = 0; s < nc; ++s) X[p * nc + s] = X[p * nc + s] * inv;
    }
  }
}

__global__ void k_update(double *X, double *dX, int64_t n, double dt) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const double d = dX[i] * dt;
    dX[i] = d;
    X[i] = X[i] + d;
  }
}

// Order-preserving map of doubles to unsigned keys (for atomic min/max).
__device__ __forceinline__ unsigned long long dkey(double v) {
  const unsigned long long b = (unsigned long long)__double_as_longlong(v);
  return (b >> 63) ? ~b : (b | 0x8000000000000000ULL);
}
__host__ __device__ inline double dkey_inv(unsigned long long k) {
  const unsigned long long b = (k >> 63) ? (k & 0x7fffffffffffffffULL) : ~k;
  double v;
  memcpy(&v, &b, sizeof(v));
  return v;
}

// stats: [0] non-finite count, [1] max row sum key, [2] min row sum key,
// [3] max component key, [4] min component key.  Row sums left to right
// (numpy's sum over a length-4 axis).
__global__ void k_oob_stats(const double *__restrict__ X, int64_t npts, int nc,
                            unsigned long long *stats) {
  unsigned long long nonfinite = 0, smax = 0, smin = ~0ULL, cmax = 0, cmin = ~0ULL;
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < npts;
       p += (int64_t)gridDim.x * blockDim.x) {
    double sum = 0.0;
    bool finite = true;
    for (int s = 0; s < nc; ++s) {
      const double v = X[p * nc + s];
      if (!isfinite(v)) {
        finite = false;
        ++nonfinite;
      } else {
        const unsigned long long k = dkey(v);
        cmax = k > cmax ? k : cmax;
        cmin = k < cmin ? k : cmin;
      }
      sum = sum + v;
    }
    if (finite) {
      const unsigned long long k = dkey(sum);
      smax = k > smax ? k : smax;
      smin = k < smin ? k : smin;
    }
  }
  if (nonfinite) atomicAdd(&stats[0], nonfinite);
  atomicMax(&stats[1], smax);
  atomicMin(&stats[2], smin);
  atomicMax(&stats[3], cmax);
  atomicMin(&stats[4], cmin);
}

static bool dims_ok(int32_t dim, const int64_t *shape, int64_t &n0, int64_t &n1, int64_t &n2) {
  if (dim < 1 || dim > 3 || !shape) return false;
  n0 = shape[0];
  n1 = dim > 1 ? shape[1] : 1;
  n2 = dim > 2 ? shape[2] : 1;
  return n0 > 0 && n1 > 0 && n2 > 0;
}

}  // namespace pf5d

using namespace pf5d;

extern "C" {

const char *pf5d_last_error(void) { return g_last_error.c_str(); }
int32_t pf5d_version(void) { return 100; }

pf5d_status pf5d_interp4d(const double *comp, int64_t npts, const double *grid, int32_t n,
                          int32_t nprops, int32_t node_stride, double resolution,
                          const double *node_coord, double max_nn_dist, double *out,
                          int64_t out_stride, uint8_t *mask, uint32_t *flags, void *stream) {
  PF5D_REQUIRE(npts >= 0, PF5D_ERR_ARG, "npts < 0");
  if (npts == 0) return PF5D_OK;
  PF5D_REQUIRE(comp && grid && node_coord && out, PF5D_ERR_ARG, "null pointer");
  PF5D_REQUIRE(nprops == NP, PF5D_ERR_ARG, "nprops must be %d (got %d)", NP, nprops);
  PF5D_REQUIRE(node_stride >= nprops && n >= 2, PF5D_ERR_ARG, "bad table geometry");
  PF5D_REQUIRE(out_stride >= nprops, PF5D_ERR_ARG, "out_stride < nprops");
  PF5D_REQUIRE(((uintptr_t)comp & 15) == 0, PF5D_ERR_ARG, "comp must be 16-byte aligned");
  Table T;
  T.grid = grid;
  T.coord = node_coord;
  T.n = n;
  T.stride = node_stride;
  T.inv_step = 1.0 / resolution;
  T.threshold = 1.0 - 4.0 * resolution - 1e-9;
  T.max_nn_dist = max_nn_dist;
  k_interp4d<<<grid_for(npts, 128), 128, 0, as_stream(stream)>>>(comp, npts, T, out, out_stride,
                                                                  mask, flags);
  PF5D_LAUNCHED();
  return PF5D_OK;
}

pf5d_status pf5d_laplacian(int32_t dim, const int64_t *shape, int32_t ncomp, const double *c,
                           double dx, double *out, void *stream) {
  int64_t n0, n1, n2;
  PF5D_REQUIRE(dims_ok(dim, shape, n0, n1, n2), PF5D_ERR_DIM,
               "Laplacian not implemented for spatial_dims=%d", dim);
  PF5D_REQUIRE(c && out && ncomp > 0, PF5D_ERR_ARG, "bad arguments");
  const double inv_dx2 = 1.0 / (dx * dx);
  const int64_t npts = n0 * n1 * n2;
  k_laplacian<<<grid_for(npts, 256), 256, 0, as_stream(stream)>>>(dim, n0, n1, n2, ncomp, c,
                                                                   inv_dx2, out);
  PF5D_LAUNCHED();
  return PF5D_OK;
}

pf5d_status pf5d_kappa_subtract(double *mu, int64_t mu_stride, double *lap, const double *kappa,
                                int64_t npts, int32_t ncomp, void *stream) {
  PF5D_REQUIRE(mu && lap && kappa && ncomp > 0 && ncomp <= 8 && mu_stride >= ncomp,
               PF5D_ERR_ARG, "bad arguments");
  if (npts <= 0) return PF5D_OK;
  Kappa k{};
  for (int s = 0; s < ncomp; ++s) k.k[s] = kappa[s];
  k_kappa_subtract<<<grid_for(npts, 256), 256, 0, as_stream(stream)>>>(mu, mu_stride, lap, k,
                                                                        npts, ncomp);
  PF5D_LAUNCHED();
  return PF5D_OK;
}

pf5d_status pf5d_divergence_from_mu(int32_t dim, const int64_t *shape, int32_t ncomp,
                                    const double *X, const double *M, int64_t m_stride,
                                    const double *mu, int64_t mu_stride, double inv_dx,
                                    double *out, void *stream) {
  int64_t n0, n1, n2;
  PF5D_REQUIRE(dims_ok(dim, shape, n0, n1, n2), PF5D_ERR_DIM,
               "Unsupported system_dim=%d. Choose 1, 2, or 3.", dim);
  PF5D_REQUIRE(ncomp == S, PF5D_ERR_ARG, "ncomp must be %d", S);
  PF5D_REQUIRE(X && M && mu && out && m_stride >= NM && mu_stride >= S, PF5D_ERR_ARG,
               "bad arguments");
  const int64_t npts = n0 * n1 * n2;
  k_divergence<<<grid_for(npts, 128), 128, 0, as_stream(stream)>>>(dim, n0, n1, n2, X, M,
                                                                   m_stride, mu, mu_stride,
                                                                   inv_dx, out);
  PF5D_LAUNCHED();
  return PF5D_OK;
}

pf5d_status pf5d_gradients_pm(int32_t dim, const int64_t *shape, int32_t ncomp, const double *c,
                              int64_t c_stride, double dx, double *gp, double *gm, void *stream) {
  int64_t n0, n1, n2;
  PF5D_REQUIRE(dims_ok(dim, shape, n0, n1, n2), PF5D_ERR_DIM,
               "Gradients not implemented for spatial_dims=%d", dim);
  PF5D_REQUIRE(c && gp && gm && ncomp > 0 && c_stride >= ncomp, PF5D_ERR_ARG, "bad arguments");
  const int64_t npts = n0 * n1 * n2;
  k_gradients_pm<<<grid_for(npts, 256), 256, 0, as_stream(stream)>>>(dim, n0, n1, n2, ncomp, c,
                                                                      c_stride, 1.0 / dx, gp, gm);
  PF5D_LAUNCHED();
  return PF5D_OK;
}

pf5d_status pf5d_fluxes_pm(int32_t dim, const int64_t *shape, int32_t ncomp, const double *X,
                           const double *M, int64_t m_stride, const double *gp, const double *gm,
                           double *fp, double *fm, void *stream) {
  int64_t n0, n1, n2;
  PF5D_REQUIRE(dims_ok(dim, shape, n0, n1, n2), PF5D_ERR_DIM,
               "Unsupported system_dim=%d. Choose 1, 2, or 3.", dim);
  PF5D_REQUIRE(ncomp == S && X && M && gp && gm && fp && fm && m_stride >= NM, PF5D_ERR_ARG,
               "bad arguments");
  const int64_t npts = n0 * n1 * n2;
  k_fluxes_pm<<<grid_for(npts, 128), 128, 0, as_stream(stream)>>>(dim, n0, n1, n2, X, M,
                                                                  m_stride, gp, gm, fp, fm);
  PF5D_LAUNCHED();
  return PF5D_OK;
}

pf5d_status pf5d_abs_max(const double *a, int64_t n, double *result, void *stream) {
  PF5D_REQUIRE(result && (a || n == 0) && n >= 0, PF5D_ERR_ARG, "bad arguments");
  double *ws = nullptr;
  pf5d_status st = absmax_workspace(&ws);
  if (st != PF5D_OK) return st;
  const unsigned blocks = n > 0 ? grid_for(n, kAbsMaxThreads) : 1;
  const unsigned nb = blocks < kAbsMaxBlocks ? blocks : kAbsMaxBlocks;
  k_absmax_partial<<<nb, kAbsMaxThreads, 0, as_stream(stream)>>>(a, n, ws);
  PF5D_LAUNCHED();
  k_absmax_final<<<1, kAbsMaxThreads, 0, as_stream(stream)>>>(ws, (int)nb, result);
  PF5D_LAUNCHED();
  return PF5D_OK;
}

pf5d_status pf5d_clamp_simplex(double *X, int64_t npts, int32_t ncomp, void *stream) {
  PF5D_REQUIRE(X && ncomp > 0 && npts >= 0, PF5D_ERR_ARG, "bad arguments");
  if (npts == 0) return PF5D_OK;
  k_clamp<<<grid_for(npts, 256), 256, 0, as_stream(stream)>>>(X, npts, ncomp);
  PF5D_LAUNCHED();
  return PF5D_OK;
}

pf5d_status pf5d_update(double *X, double *dXdt, int64_t n, double dt, void *stream) {
  PF5D_REQUIRE(X && dXdt && n >= 0, PF5D_ERR_ARG, "bad arguments");
  if (n == 0) return PF5D_OK;
  k_update<<<grid_for(n, 256), 256, 0, as_stream(stream)>>>(X, dXdt, n, dt);
  PF5D_LAUNCHED();
  return PF5D_OK;
}

pf5d_status pf5d_oob_stats(const double *X, int64_t npts, int32_t ncomp, double *stats,
                           void *stream) {
  PF5D_REQUIRE(X && stats && ncomp > 0 && npts > 0, PF5D_ERR_ARG, "bad arguments");
  cudaStream_t s = as_stream(stream);
  unsigned long long init[5] = {0ULL, 0ULL, ~0ULL, 0ULL, ~0ULL};
  unsigned long long *d = nullptr;
  PF5D_CUDA(cudaMallocAsync(&d, sizeof(init), s));
  PF5D_CUDA(cudaMemcpyAsync(d, init, sizeof(init), cudaMemcpyHostToDevice, s));
  k_oob_stats<<<grid_for(npts, 256), 256, 0, s>>>(X, npts, ncomp, d);
  PF5D_LAUNCHED();
  unsigned long long h[5];
  PF5D_CUDA(cudaMemcpyAsync(h, d, sizeof(h), cudaMemcpyDeviceToHost, s));
  PF5D_CUDA(cudaFreeAsync(d, s));
  PF5D_CUDA(cudaStreamSynchronize(s));
  stats[0] = (double)h[0];
  stats[1] = dkey_inv(h[1]);
  stats[2] = dkey_inv(h[2]);
  stats[3] = dkey_inv(h[3]);
  stats[4] = dkey_inv(h[4]);
  return PF5D_OK;
}

double pf5d_adaptive_dt(double dt_current, double xdotmax, double ctld, double t_cfl,
                        double lower_limit, double upper_limit, double max_change_factor) {
  return adaptive_dt(dt_current, xdotmax, ctld, t_cfl, lower_limit, upper_limit,
                     max_change_factor);
}

}  // extern "C"
