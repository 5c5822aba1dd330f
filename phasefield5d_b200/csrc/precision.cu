// precision.cu -- FP32-compensated form of the step loop (the "precision
// form").  Same dataflow and tiling as the FP64 stepper (stepper.cu):
//   cuFFT R2C of the misfit -> B(k)/N multiply -> cuFFT C2R -> fused rate
//   kernel (FP32 interpolation, Laplacian, mu, one flux per face,
//   divergence, a max|dX/dt| slot per block) -> k32_dt (one block: the
//   FP64 dt controller) -> compensated update + clamp + next misfit +
//   out-of-bounds test,
// replayed from CUDA graphs.
//
// Numerics:
//   * the field is D = X - X0 as an FP32 pair (hi, lo); the update adds
//     dt*dX/dt with TwoSum and renormalises, so rounding does not
//     accumulate over thousands of steps;
//   * the table stores mu - mu(X0) (and M) in FP32, so mu gradients are
//     differences of small numbers;
//   * cell fractions come from a host FP64 split of X0/res into integer and
//     fraction plus the FP32 deviation D/res;
//   * FP64: closure X_Fe = 1 - sum X (face flux), linear-region and simplex
//     sums, dt controller, mass/mean reductions.  The k = 0 elastic mode is
//     exactly zero because B(0) = 0.
// Compiled with FMA contraction allowed; the TwoSum update uses explicit
// round-to-nearest intrinsics so it is never contracted.
#include <algorithm>
#include <cstring>
#include <map>
#include <vector>

#include <cuda_pipeline_primitives.h>
#include <cufft.h>

#include "pf5d_device.cuh"
#include "pf5d_fft.h"
#include "pf5d_fp32c.h"
#include "pf5d_fp32c.cuh"
#include "pf5d_host.h"
#include "pf5d_tiles.cuh"
#include "pf5d_window.cuh"

namespace pf5d {

// ------------------------------------------------------------------------
// Rate kernels (same tiling as the FP64 kernels)
// ------------------------------------------------------------------------

template <int TX, int TY, int MINB, bool WIN, int SORT = 0, bool SPLIT = false,
          bool PERPOINT = false>
__global__ void __launch_bounds__(TX * TY, MINB) k32_rate_tile2d(Rate32 P) {
  pdl_wait();
  if (P.st->halt) return;
  extern __shared__ float4 sm4[];
  const int tid = threadIdx.y * TX + threadIdx.x;
  unsigned flags = 0;
  const float vmax = tile2d32_body<TX, TY, WIN, SORT, SPLIT, PERPOINT>(P, blockIdx.x, blockIdx.y,
                                                                      sm4, &flags, tid);
  raise_rate_flags(P.st, flags);
  finish_rate32(P, vmax, Tile2dSmem32<TX, TY, SORT>::red(sm4));
}

template <int TX, int TY, int SORT = 0>
constexpr size_t tile2d32_smem() {
  return Tile2dSmem32<TX, TY, SORT>::bytes;
}

template <int TX, int TY, int MINB, bool WIN, int SORT = 0>
__global__ void __launch_bounds__(TX * TY, MINB) k32_rate_march3d(Rate32 P, int zc) {
  using G = PlaneGeom<TX, TY>;
  pdl_wait();
  if (P.st->halt) return;
  extern __shared__ float4 sm4[];
  float4 *win = sm4;
  double *red = reinterpret_cast<double *>(win + kWinNodes32 * 3);
  float *Xs = reinterpret_cast<float *>(red + G::NT / 32);      // [3][S][PX]
  float *Ms = Xs + 3 * S * G::PX;                                // [2][NPM][PM]
  float *Fx = Ms + 2 * NPM * G::PM;
  float *Fy = Fx + S * G::NFX;
  int *wred = reinterpret_cast<int *>(Fy + S * G::NFY);
  int *win_lo = wred + S * (G::NT / 32);
  int *wx = win_lo + S + 1;
  int *wy = wx + G::HX;
  SortScratch32 ss{};
  if constexpr (SORT) ss = SortBytes32<TX, TY>::carve(wy + G::HY);
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
  const int x0 = blockIdx.x * TX, y0 = blockIdx.y * TY;
  const int zb = blockIdx.z * zc;
  const int ze = min(zb + zc, P.nz);
  const int64_t plane = (int64_t)P.ny * P.nx;
  unsigned flags = 0;
  if (tid == 0) win_lo[S] = 0;
  for (int i = tid; i < G::HX + G::HY; i += G::NT) {
    if (i < G::HX) wx[i] = wrap_any(x0 + i - 2, P.nx);
    else wy[i - G::HX] = wrap_any(y0 + (i - G::HX) - 2, P.ny);
  }
  auto xplane = [&](int z) { return Xs + ((z - zb + 3) % 3) * S * G::PX; };
  auto mplane = [&](int z) { return Ms + ((z - zb + 2) & 1) * NPM * G::PM; };
  auto load_x = [&](int z) {
    load_plane32<TX, TY>(P.D, (int64_t)wrap_any(z, P.nz) * plane, wx, wy, P.nx, xplane(z), tid);
  };
  auto compute_mu = [&](int z, bool interior_only) {
    mu_plane32<TX, TY, 3, WIN, SORT>(P, xplane(z - 1), xplane(z), xplane(z + 1), mplane(z),
                                     (int64_t)wrap_any(z, P.nz) * plane, wx, wy, interior_only,
                                     win, wred, win_lo, &flags, tid, ss);
  };
  const int pX = (ty + 2) * G::HX + (tx + 2);
  const int pM = (ty + 1) * G::MX + (tx + 1);
  const bool in_tile = (x0 + tx < P.nx) && (y0 + ty < P.ny);
  __syncthreads();
  load_x(zb - 2);
  load_x(zb - 1);
  load_x(zb);
  __syncthreads();
  compute_mu(zb - 1, true);
  __syncthreads();
  load_x(zb + 1);
  __syncthreads();
  compute_mu(zb, false);
  __syncthreads();
  float Jm[S];
  face32_between<G::PX, G::PM>(P, xplane(zb - 1), mplane(zb - 1), pX, pM, xplane(zb), mplane(zb),
                               pX, pM, Jm);
  float vmax = 0.f;
  for (int z = zb; z < ze; ++z) {
    __syncthreads();
    load_x(z + 2);
    __syncthreads();
    compute_mu(z + 1, false);
    __syncthreads();
    float Jz[S];
    face32_between<G::PX, G::PM>(P, xplane(z), mplane(z), pX, pM, xplane(z + 1), mplane(z + 1),
                                 pX, pM, Jz);
    plane_faces32<TX, TY>(P, xplane(z), mplane(z), Fx, Fy, tid);
    __syncthreads();
    if (in_tile) {
      float out[S];
#pragma unroll
      for (int c = 0; c < S; ++c) {
        const float ay = __fsub_rn(Fy[c * G::NFY + (ty + 1) * TX + tx], Fy[c * G::NFY + ty * TX + tx]);
        const float ax = __fsub_rn(Fx[c * G::NFX + ty * (TX + 1) + tx + 1],
                                   Fx[c * G::NFX + ty * (TX + 1) + tx]);
        out[c] = __fmul_rn(__fadd_rn(__fadd_rn(__fsub_rn(Jz[c], Jm[c]), ay), ax), P.flux_scale);
      }
      store_rate(P.dX, (int64_t)z * plane + (int64_t)(y0 + ty) * P.nx + (x0 + tx), out, vmax);
    }
#pragma unroll
    for (int c = 0; c < S; ++c) Jm[c] = Jz[c];
  }
  raise_rate_flags(P.st, flags);
  finish_rate32(P, vmax, red);
}

template <int TX, int TY, int SORT = 0>
constexpr size_t march3d32_smem() {
  using G = PlaneGeom<TX, TY>;
  return Smem32Tail<TX, TY>::bytes +
         (3 * S * G::PX + 2 * NPM * G::PM + S * G::NFX + S * G::NFY) * sizeof(float) +
         (SORT ? SortBytes32<TX, TY>::bytes : 0);
}

template <int TX>
__global__ void __launch_bounds__(TX) k32_rate_1d(Rate32 P) {
  pdl_wait();
  if (P.st->halt) return;
  constexpr int HX = TX + 4, MX = TX + 2;
  __shared__ float Xs[S][HX];
  __shared__ float Ms[NPM][MX];
  __shared__ float Fx[S][TX + 1];
  __shared__ double red[(TX + 31) / 32];
  const int tx = threadIdx.x;
  const int x0 = blockIdx.x * TX;
  const int n = P.nx;
  unsigned flags = 0;
  for (int pos = tx; pos < HX; pos += TX) {
    const float4 v = __ldg(P.D + wrap_any(x0 + pos - 2, n));
    Xs[0][pos] = v.x;
    Xs[1][pos] = v.y;
    Xs[2][pos] = v.z;
    Xs[3][pos] = v.w;
  }
  __syncthreads();
  for (int pos = tx; pos < MX; pos += TX) {
    const int px = pos + 1;
    float d[S], lap[S];
#pragma unroll
    for (int c = 0; c < S; ++c) {
      d[c] = Xs[c][px];
      const float nb[2] = {Xs[c][px + 1], Xs[c][px - 1]};
      lap[c] = lap32<2>(nb, d[c], P.inv_dx2);
    }
    const float spv = P.sp ? __ldg(P.sp + wrap_any(x0 + pos - 1, n)) : 0.f;
    float v[NPM];
    chem32(P, d, lap, spv, nullptr, nullptr, v, &flags);
#pragma unroll
    for (int r = 0; r < NPM; ++r) Ms[r][pos] = v[r];
  }
  __syncthreads();
  for (int f = tx; f < TX + 1; f += TX) {
    float J[S];
    face32_between<HX, MX>(P, &Xs[0][0], &Ms[0][0], f + 1, f, &Xs[0][0], &Ms[0][0], f + 2, f + 1,
                           J);
#pragma unroll
    for (int c = 0; c < S; ++c) Fx[c][f] = J[c];
  }
  __syncthreads();
  float vmax = 0.f;
  if (x0 + tx < n) {
    float out[S];
#pragma unroll
    for (int c = 0; c < S; ++c) out[c] = (Fx[c][tx + 1] - Fx[c][tx]) * P.flux_scale;
    store_rate(P.dX, x0 + tx, out, vmax);
  }
  raise_rate_flags(P.st, flags);
  finish_rate32(P, vmax, red);
}

// ------------------------------------------------------------------------
// Compensated update, clamp, next misfit, out-of-bounds test
// ------------------------------------------------------------------------
struct Update32 {
  float4 *hi, *lo;
  const float4 *dX;
  int64_t npts;
  StepState32 *st;
  double x0[S];
  double sum_x0;
  float lvec[S];
  float *s;          // next misfit or nullptr
  int oob_interval;
};

__global__ void k32_update(Update32 U) {
  pdl_wait();
  StepState32 *st = U.st;
  if (st->halt) return;
  const float dtf = (float)st->dt;
  const bool check = U.oob_interval > 0 && (st->step % U.oob_interval) == 0;
  unsigned f = 0;
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < U.npts;
       p += (int64_t)gridDim.x * blockDim.x) {
    const float4 H = U.hi[p], L = U.lo[p], R = U.dX[p];
    float h[S] = {H.x, H.y, H.z, H.w}, l[S] = {L.x, L.y, L.z, L.w};
    const float r[S] = {R.x, R.y, R.z, R.w};
#pragma unroll
    for (int c = 0; c < S; ++c) comp_add(h[c], l[c], __fmul_rn(dtf, r[c]));
    double dd[S], dsum = 0.0;
#pragma unroll
    for (int c = 0; c < S; ++c) {
      dd[c] = (double)h[c] + (double)l[c];
      dsum = dsum + dd[c];
    }
    const double total = U.sum_x0 + dsum;
    if (total > 1.0) {                 // clamp_simplex on X = X0 + D, in FP64
      const double inv = 1.0 / total;
#pragma unroll
      for (int c = 0; c < S; ++c) {
        const double dn = (U.x0[c] + dd[c]) * inv - U.x0[c];
        h[c] = (float)dn;
        l[c] = (float)(dn - (double)h[c]);
        dd[c] = (double)h[c] + (double)l[c];
      }
    }
    U.hi[p] = make_float4(h[0], h[1], h[2], h[3]);
    U.lo[p] = make_float4(l[0], l[1], l[2], l[3]);
    if (U.s) {
      float acc = 0.f;
#pragma unroll
      for (int c = 0; c < S; ++c) acc = fmaf(h[c] + l[c], U.lvec[c], acc);
      U.s[p] = acc;
    }
    if (check) {
      double x[S];
#pragma unroll
      for (int c = 0; c < S; ++c) x[c] = U.x0[c] + dd[c];
      f |= oob_flags_x(x);
    }
  }
  raise32(st, f);
}

__global__ void k32_split(const double *__restrict__ X, int64_t npts, Update32 U) {
  unsigned f = 0;
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < npts;
       p += (int64_t)gridDim.x * blockDim.x) {
    float h[S], l[S];
    double x[S];
#pragma unroll
    for (int c = 0; c < S; ++c) {
      x[c] = X[4 * p + c];
      const double d = x[c] - U.x0[c];
      h[c] = (float)d;
      l[c] = (float)(d - (double)h[c]);
    }
    U.hi[p] = make_float4(h[0], h[1], h[2], h[3]);
    U.lo[p] = make_float4(l[0], l[1], l[2], l[3]);
    if (U.s) {
      float acc = 0.f;
#pragma unroll
      for (int c = 0; c < S; ++c) acc = fmaf(h[c] + l[c], U.lvec[c], acc);
      U.s[p] = acc;
    }
    if (U.oob_interval > 0) f |= oob_flags_x(x);
  }
  raise32(U.st, f);
}

__global__ void k32_join(const float4 *__restrict__ hi, const float4 *__restrict__ lo,
                         int64_t npts, Update32 U, double *__restrict__ X) {
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < npts;
       p += (int64_t)gridDim.x * blockDim.x) {
    const float4 H = hi[p], L = lo[p];
    const float h[S] = {H.x, H.y, H.z, H.w}, l[S] = {L.x, L.y, L.z, L.w};
#pragma unroll
    for (int c = 0; c < S; ++c) X[4 * p + c] = U.x0[c] + ((double)h[c] + (double)l[c]);
  }
}

constexpr int kMassBlocks = 512;

// FP64 per-component sums of X = X0 + hi + lo; two passes, deterministic.
__global__ void k32_mass_partial(const float4 *__restrict__ hi, const float4 *__restrict__ lo,
                                 int64_t npts, double *partial) {
  __shared__ double red[S][8];
  double acc[S] = {0.0, 0.0, 0.0, 0.0};
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < npts;
       p += (int64_t)gridDim.x * blockDim.x) {
    const float4 H = hi[p], L = lo[p];
    acc[0] += (double)H.x + (double)L.x;
    acc[1] += (double)H.y + (double)L.y;
    acc[2] += (double)H.z + (double)L.z;
    acc[3] += (double)H.w + (double)L.w;
  }
#pragma unroll
  for (int c = 0; c < S; ++c) {
    double v = acc[c];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) red[c][threadIdx.x >> 5] = v;
  }
  __syncthreads();
  if (threadIdx.x < S) {
    double v = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) v += red[threadIdx.x][w];
    partial[blockIdx.x * S + threadIdx.x] = v;
  }
}

__global__ void k32_mass_final(const double *partial, int nparts, double *out) {
  if (threadIdx.x < S) {
    double v = 0.0;
    for (int b = 0; b < nparts; ++b) v += partial[b * S + threadIdx.x];
    out[threadIdx.x] = v;
  }
}

// ------------------------------------------------------------------------
// Split rate evaluation, first kernel: mu/M and the closure X_Fe at every
// point of a 1D/2D/3D field into the split buffers (mm_mu, mm_m, mm_f).
//
// A block of 256 threads takes a brick of 256 K points (32 x 8 x K in 3D,
// 32 x 8K in 2D, 256K in 1D) in six phases:
//   1. per point: Laplacian (neighbour order +axis0, -axis0, ...), the mu
//      offset s' l - kappa lap, the FP64 closure, the table cell and its
//      fractions (the deviation itself for points outside the linear region);
//   2. counting sort of the points by a hash of their exact cell (bin 255
//      holds the points outside the linear region);
//   3. each linear bin's run is cut into work items of up to K consecutive
//      points;
//   4. a thread evaluates a work item: the 16 corner nodes of the item's
//      cell are loaded once and accumulated into every point of the item
//      with the point's own weights, so the table traffic per point drops
//      K-fold (the lanes of a warp hold neighbouring items, mostly of the
//      same cell, so the loads are broadcasts).  A point whose exact cell
//      differs from the item's first (a hash collision) is set aside;
//   5. the points set aside and those outside the linear region (nearest
//      table row), one per thread;
//   6. the block's outputs are stored coalesced.
// Per point the block keeps three float4 in shared memory (point-major, so a
// thread reads or writes a point's values with vector loads): the cell
// fractions (or the deviation d outside the linear region), the mu offset,
// and (cell, X_Fe); the outputs overwrite them as (mu), (M_Fe, M_1..3),
// (M_4, X_Fe).  Every value is formed by the same routines, in the same
// order, as in the fused kernels (weights32 / corner_acc32, mu_offset32,
// dsum32).
// ------------------------------------------------------------------------
constexpr int kChemThreads = 256;

template <int DIM, int K>
struct ChemGeom {
  static constexpr int NPB = kChemThreads * K;                     // points per block
  static constexpr int BX = DIM == 1 ? NPB : 32;
  static constexpr int BY = DIM == 1 ? 1 : (DIM == 2 ? 8 * K : 8);
  static constexpr int BZ = DIM == 3 ? K : 1;
  static constexpr int NITEMS = NPB / K + 256;                      // upper bound on items
  // pio[3][NPB] float4 (point-major); items[NITEMS] u32; order, prank, left
  // [NPB] u16; skey, pkey [NPB] u8; hist / cnt / ibase [256] int; wsum, nleft
  static constexpr size_t smem = (size_t)3 * 16 * NPB + NITEMS * 4 + 3 * NPB * 2 + 2 * NPB +
                                 3 * 256 * 4 + 16 * 4;
};

__device__ __forceinline__ int cell_key32(const int ii[S]) {
  return (int)((unsigned)(41 * ii[0] + 13 * ii[1] + 5 * ii[2] + ii[3]) % 255u);
}

template <int DIM, int K, int MINB>
__global__ void __launch_bounds__(kChemThreads, MINB) k32_chem(Rate32 P) {
  using G = ChemGeom<DIM, K>;
  constexpr int NT = kChemThreads, NPB = G::NPB;
  extern __shared__ float4 sm4[];
  float4 *pio = sm4;                                                   // 3 per point
  unsigned *items = reinterpret_cast<unsigned *>(pio + 3 * NPB);
  unsigned short *order = reinterpret_cast<unsigned short *>(items + G::NITEMS);
  unsigned short *prank = order + NPB;
  unsigned short *left = prank + NPB;
  unsigned char *skey = reinterpret_cast<unsigned char *>(left + NPB);
  unsigned char *pkey = skey + NPB;
  int *hist = reinterpret_cast<int *>(pkey + NPB);                     // NPB % 4 == 0
  int *cnt = hist + 256;
  int *ibase = cnt + 256;
  int *wsum = ibase + 256;
  int *nleft = wsum + 12;
  pdl_wait();
  if (P.st->halt) return;
  const int tid = threadIdx.x;
  const Table32 &T = P.T;
  const int64_t plane = (int64_t)P.ny * P.nx;
  hist[tid] = 0;
  if (tid == 0) *nleft = 0;
  __syncthreads();
  // 1. per-point inputs
#pragma unroll 1
  for (int j = 0; j < K; ++j) {
    const int q = tid + j * NT;
    const int qx = q % G::BX, qy = (q / G::BX) % G::BY, qz = q / (G::BX * G::BY);
    const int x = blockIdx.x * G::BX + qx, y = blockIdx.y * G::BY + qy, z = blockIdx.z * G::BZ + qz;
    prank[q] = 0xFFFFu;
    if (x >= P.nx || y >= P.ny || z >= P.nz) continue;
    const int64_t zo = (int64_t)z * plane, g = zo + (int64_t)y * P.nx + x;
    auto ld = [&](int64_t gi, float v[S]) {
      const float4 a = __ldg(P.D + gi);
      v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
    };
    constexpr int NB = 2 * DIM;
    float d[S], nb[NB][S];
    ld(g, d);
    int k = 0;
    if (DIM == 3) {
      const int zp = z + 1 == P.nz ? 0 : z + 1, zm = z == 0 ? P.nz - 1 : z - 1;
      ld((int64_t)zp * plane + (int64_t)y * P.nx + x, nb[k++]);
      ld((int64_t)zm * plane + (int64_t)y * P.nx + x, nb[k++]);
    }
    if (DIM >= 2) {
      const int yp = y + 1 == P.ny ? 0 : y + 1, ym = y == 0 ? P.ny - 1 : y - 1;
      ld(zo + (int64_t)yp * P.nx + x, nb[k++]);
      ld(zo + (int64_t)ym * P.nx + x, nb[k++]);
    }
    const int xp = x + 1 == P.nx ? 0 : x + 1, xm = x == 0 ? P.nx - 1 : x - 1;
    ld(zo + (int64_t)y * P.nx + xp, nb[k++]);
    ld(zo + (int64_t)y * P.nx + xm, nb[k]);
    float lap[S], off[S];
#pragma unroll
    for (int c = 0; c < S; ++c) {
      float n[NB];
#pragma unroll
      for (int i = 0; i < NB; ++i) n[i] = nb[i][c];
      lap[c] = lap32<NB>(n, d[c], P.inv_dx2);
    }
    mu_offset32(P, lap, P.sp ? __ldg(P.sp + g) : 0.f, off);
    const double sd = dsum32(d);
    int ii[S];
    float tt[S];
    int cell = -1, key = 255;
    if (cell32(T, d, sd, ii, tt)) {
      cell = ((ii[0] * T.n + ii[1]) * T.n + ii[2]) * T.n + ii[3];
      key = cell_key32(ii);
    } else {
#pragma unroll
      for (int c = 0; c < S; ++c) tt[c] = d[c];
    }
    pio[3 * q] = make_float4(tt[0], tt[1], tt[2], tt[3]);
    pio[3 * q + 1] = make_float4(off[0], off[1], off[2], off[3]);
    pio[3 * q + 2] = make_float4(__int_as_float(cell), (float)(P.c_fe - sd), 0.f, 0.f);
    pkey[q] = (unsigned char)key;
    prank[q] = (unsigned short)atomicAdd(&hist[key], 1);
  }
  __syncthreads();
  // 2. counting sort by cell key
  cnt[tid] = hist[tid];
  const int nvalid = block_exclusive_scan<256, NT>(hist, wsum, tid);
  for (int q = tid; q < NPB; q += NT) {
    if (prank[q] == 0xFFFFu) continue;
    const int b = pkey[q], s = hist[b] + prank[q];
    order[s] = (unsigned short)q;
    skey[s] = (unsigned char)b;
  }
  // 3. work items: runs of up to K points of one linear bin
  ibase[tid] = tid == 255 ? 0 : (cnt[tid] + K - 1) / K;
  const int nitems = block_exclusive_scan<256, NT>(ibase, wsum, tid);
  const int lin_end = nvalid - cnt[255];            // bin 255 (nearest row) sorts last
  for (int s = tid; s < lin_end; s += NT) {
    const int b = skey[s], r = s - hist[b];
    if (r % K == 0) items[ibase[b] + r / K] = (unsigned)s | ((unsigned)min(K, cnt[b] - r) << 16);
  }
  __syncthreads();
  // 4. the work items
  const float4 *g4 = reinterpret_cast<const float4 *>(T.grid);
  const int64_t s3 = 3, s2 = 3 * (int64_t)T.n, s1 = s2 * T.n, s0 = s1 * T.n;
  for (int it = tid; it < nitems; it += NT) {
    const unsigned e = items[it];
    const int s = (int)(e & 0xFFFFu), m = (int)(e >> 16);
    int q[K];
    bool use[K];
    Weights32 W[K];
    int cell0 = 0;
#pragma unroll
    for (int j = 0; j < K; ++j) {
      q[j] = j < m ? (int)order[s + j] : 0;
      const int cj = __float_as_int(pio[3 * q[j] + 2].x);
      if (j == 0) cell0 = cj;
      use[j] = j < m && cj == cell0;
      if (j < m && !use[j]) left[atomicAdd(nleft, 1)] = (unsigned short)q[j];
      const float4 t4 = pio[3 * q[j]];
      const float tt[S] = {t4.x, t4.y, t4.z, t4.w};
      W[j] = weights32(tt);
    }
    float acc[K][NP];
    const float4 *base = g4 + (int64_t)cell0 * 3;
#pragma unroll
    for (int c = 0; c < 16; ++c) {
      const int b0 = (c >> 3) & 1, b1 = (c >> 2) & 1, b2 = (c >> 1) & 1, b3 = c & 1;
      const float4 *node = base + b0 * s0 + b1 * s1 + b2 * s2 + b3 * s3;
      const float4 a = __ldg(node), b = __ldg(node + 1), f = __ldg(node + 2);
#pragma unroll
      for (int j = 0; j < K; ++j) corner_acc32(c, W[j].wa[c >> 2] * W[j].wb[c & 3], a, b, f, acc[j]);
    }
    // mu = table value + offset; rows in chem32's order (X_Fe stays in row 9)
#pragma unroll
    for (int j = 0; j < K; ++j) {
      if (!use[j]) continue;
      float4 *o = pio + 3 * q[j];
      const float4 off = o[1];
      o[0] = make_float4(acc[j][0] + off.x, acc[j][1] + off.y, acc[j][2] + off.z, acc[j][3] + off.w);
      o[1] = make_float4(acc[j][4], acc[j][5], acc[j][6], acc[j][7]);
      o[2].x = acc[j][8];
    }
  }
  __syncthreads();
  // 5. points set aside and points outside the linear region, one per thread
  unsigned flags = 0;
  const int nnn = cnt[255], nl = nnn + *nleft;
  for (int l = tid; l < nl; l += NT) {
    const int q = l < nnn ? (int)order[lin_end + l] : (int)left[l - nnn];
    float4 *o = pio + 3 * q;
    const int cell = __float_as_int(o[2].x);
    const float4 a4 = o[0];
    const float a[S] = {a4.x, a4.y, a4.z, a4.w};
    float v[NP];
    if (cell < 0) nearest_row32(T, a, v, &flags);
    else interp_nodes32(g4 + (int64_t)cell * 3, (int)s0, (int)s1, (int)s2, (int)s3, a, v);
    const float4 off = o[1];
    o[0] = make_float4(v[0] + off.x, v[1] + off.y, v[2] + off.z, v[3] + off.w);
    o[1] = make_float4(v[4], v[5], v[6], v[7]);
    o[2].x = v[8];
  }
  raise_rate_flags(P.st, flags);
  __syncthreads();
  // 6. coalesced stores
#pragma unroll 1
  for (int j = 0; j < K; ++j) {
    const int q = tid + j * NT;
    const int qx = q % G::BX, qy = (q / G::BX) % G::BY, qz = q / (G::BX * G::BY);
    const int x = blockIdx.x * G::BX + qx, y = blockIdx.y * G::BY + qy, z = blockIdx.z * G::BZ + qz;
    if (x >= P.nx || y >= P.ny || z >= P.nz) continue;
    const int64_t g = (int64_t)z * plane + (int64_t)y * P.nx + x;
    const float4 a = pio[3 * q], b = pio[3 * q + 1], c = pio[3 * q + 2];
    P.mm_mu[g] = a;
    P.mm_m[g] = make_float4(b.y, b.z, b.w, c.x);
    P.mm_f[g] = make_float2(b.x, c.y);
  }
}

template <int DIM, int K, int MINB>
void chem32_attrs() {
  cudaFuncSetAttribute(k32_chem<DIM, K, MINB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)ChemGeom<DIM, K>::smem);
}

template <int DIM, int K, int MINB>
void launch_chem32(cudaStream_t s, const Rate32 &P) {
  using G = ChemGeom<DIM, K>;
  const dim3 g((unsigned)((P.nx + G::BX - 1) / G::BX), (unsigned)((P.ny + G::BY - 1) / G::BY),
               (unsigned)((P.nz + G::BZ - 1) / G::BZ));
  launch_pdl(k32_chem<DIM, K, MINB>, g, dim3(kChemThreads), G::smem, s, P);
}

// ------------------------------------------------------------------------
// Split rate evaluation, second kernel in 3D: face fluxes and divergence of
// a TX x TY plane tile marching along axis 0, from the split buffers.  Each
// plane position of the tile and its 1-cell halo (corners skipped) is
// staged as it is stored -- float4 D, float4 mu, float4 M, float2 (M_Fe,
// X_Fe) -- by cp.async into a three-slot ring, so plane z+2 is in flight
// while plane z is evaluated.  PERPOINT: each point evaluates its four
// in-plane faces (a face by both of its cells, with the same operands and
// operation order); otherwise each in-plane face is evaluated once into
// shared buffers.  Same face routine and divergence order as the fused
// marching kernel.
// ------------------------------------------------------------------------
template <int TX, int TY>
struct Flux3Geom {
  static constexpr int MX = TX + 2, MY = TY + 2, PM = MX * MY, NT = TX * TY;
  static constexpr int NFX = TY * (TX + 1), NFY = (TY + 1) * TX;
  static constexpr size_t slot = (size_t)PM * (3 * 16 + 8);       // bytes per ring slot
  static constexpr size_t smem(bool perpoint) {
    return 3 * slot + (perpoint ? 0 : (size_t)(NFX + NFY) * 16) + (NT / 32) * 8 +
           (MX + MY) * 4;
  }
};

template <int TX, int TY, int MINB, bool PERPOINT>
__global__ void __launch_bounds__(TX * TY, MINB) k32_flux3(Rate32 P, int zc) {
  using G = Flux3Geom<TX, TY>;
  static_assert(G::slot % 16 == 0, "ring slots must stay 16-byte aligned");
  pdl_wait();
  if (P.st->halt) return;
  extern __shared__ float4 sm4[];
  // ring slot r: D[PM], mu[PM], M[PM] (float4) then F[PM] (float2)
  float4 *ring = sm4;
  float4 *Fx = reinterpret_cast<float4 *>(reinterpret_cast<char *>(sm4) + 3 * G::slot);
  float4 *Fy = Fx + (PERPOINT ? 0 : G::NFX);
  double *red = reinterpret_cast<double *>(Fy + (PERPOINT ? 0 : G::NFY));
  int *wx = reinterpret_cast<int *>(red + G::NT / 32);
  int *wy = wx + G::MX;
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
  const int x0 = blockIdx.x * TX, y0 = blockIdx.y * TY;
  const int zb = blockIdx.z * zc;
  const int ze = min(zb + zc, P.nz);
  const int64_t plane = (int64_t)P.ny * P.nx;
  for (int i = tid; i < G::MX + G::MY; i += G::NT) {
    if (i < G::MX) wx[i] = wrap_any(x0 + i - 1, P.nx);
    else wy[i - G::MX] = wrap_any(y0 + (i - G::MX) - 1, P.ny);
  }
  __syncthreads();
  auto sD = [&](int z) { return ring + ((z - zb + 3) % 3) * (G::slot / 16); };
  auto sMu = [&](int z) { return sD(z) + G::PM; };
  auto sM = [&](int z) { return sD(z) + 2 * G::PM; };
  auto sF = [&](int z) { return reinterpret_cast<float2 *>(sD(z) + 3 * G::PM); };
  auto issue = [&](int z, bool interior_only) {
    const int64_t zoff = (int64_t)wrap_any(z, P.nz) * plane;
    float4 *d = sD(z), *mu = sMu(z), *m = sM(z);
    float2 *f = sF(z);
    for (int pos = tid; pos < G::PM; pos += G::NT) {
      const int my = pos / G::MX, mx = pos - my * G::MX;
      const bool ex = (mx == 0 || mx == G::MX - 1), ey = (my == 0 || my == G::MY - 1);
      if (interior_only ? (ex || ey) : (ex && ey)) continue;
      const int64_t g = zoff + (int64_t)wy[my] * P.nx + wx[mx];
      __pipeline_memcpy_async(d + pos, P.D + g, 16);
      __pipeline_memcpy_async(mu + pos, P.mm_mu + g, 16);
      __pipeline_memcpy_async(m + pos, P.mm_m + g, 16);
      __pipeline_memcpy_async(f + pos, P.mm_f + g, 8);
    }
    __pipeline_commit();
  };
  auto face = [&](int zl, int pl, int zh, int ph) {
    return face_flux32(P, sD(zl)[pl], sMu(zl)[pl], sM(zl)[pl], sF(zl)[pl], sD(zh)[ph],
                       sMu(zh)[ph], sM(zh)[ph], sF(zh)[ph]);
  };
  const int p = (ty + 1) * G::MX + (tx + 1);
  const bool in_tile = (x0 + tx < P.nx) && (y0 + ty < P.ny);
  issue(zb - 1, true);
  issue(zb, false);
  issue(zb + 1, false);
  __pipeline_wait_prior(1);
  __syncthreads();
  float4 Jm = face(zb - 1, p, zb, p);
  float vmax = 0.f;
  for (int z = zb; z < ze; ++z) {
    __pipeline_wait_prior(0);          // plane z+1 copied (this thread's part)
    __syncthreads();                   // ... and every thread's; slot of z-1 free
    if (z + 2 <= ze) issue(z + 2, false);
    const float4 Jz = face(z, p, z + 1, p);
    float4 jyp, jym, jxp, jxm;
    if constexpr (PERPOINT) {
      jyp = face(z, p, z, p + G::MX);
      jym = face(z, p - G::MX, z, p);
      jxp = face(z, p, z, p + 1);
      jxm = face(z, p - 1, z, p);
    } else {
      for (int f = tid; f < G::NFX + G::NFY; f += G::NT) {
        if (f < G::NFX) {
          const int fy = f / (TX + 1), fx = f - fy * (TX + 1);
          const int pl = (fy + 1) * G::MX + fx;
          Fx[f] = face(z, pl, z, pl + 1);
        } else {
          const int f2 = f - G::NFX;
          const int fy = f2 / TX, fx = f2 - fy * TX;
          const int pl = fy * G::MX + (fx + 1);
          Fy[f2] = face(z, pl, z, pl + G::MX);
        }
      }
      __syncthreads();
      jyp = Fy[(ty + 1) * TX + tx];
      jym = Fy[ty * TX + tx];
      jxp = Fx[ty * (TX + 1) + tx + 1];
      jxm = Fx[ty * (TX + 1) + tx];
    }
    if (in_tile) {
      const float a[S] = {Jz.x - Jm.x, Jz.y - Jm.y, Jz.z - Jm.z, Jz.w - Jm.w};
      const float ay[S] = {jyp.x - jym.x, jyp.y - jym.y, jyp.z - jym.z, jyp.w - jym.w};
      const float ax[S] = {jxp.x - jxm.x, jxp.y - jxm.y, jxp.z - jxm.z, jxp.w - jxm.w};
      float out[S];
#pragma unroll
      for (int c = 0; c < S; ++c) out[c] = ((a[c] + ay[c]) + ax[c]) * P.flux_scale;
      store_rate(P.dX, (int64_t)z * plane + (int64_t)(y0 + ty) * P.nx + (x0 + tx), out, vmax);
    }
    Jm = Jz;
  }
  __pipeline_wait_prior(0);
  finish_rate32(P, vmax, red);
}

// The dt controller after a rate launch of `nparts` blocks: a block-wide
// max over the slots, then the FP64 rule in thread 0.
constexpr int kDt32Threads = 1024;
__global__ void __launch_bounds__(kDt32Threads) k32_dt(Rate32 P, int nparts) {
  __shared__ double red[kDt32Threads / 32];
  pdl_wait();
  StepState32 *st = P.st;
  if (st->halt) return;
  double m = 0.0;
  for (int i = threadIdx.x; i < nparts; i += kDt32Threads) m = fmax(m, P.partial[i]);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < kDt32Threads / 32; ++w) m = fmax(m, red[w]);
    double dt = st->dt;
    if (P.adaptive) dt = adaptive_dt(dt, m, P.ctld, P.t_cfl, P.lower, P.upper, P.factor);
    st->dt = dt;
    st->time = st->time + dt;
    st->xdotmax = m;
    st->step = st->step + 1;
  }
}

// The 1D elastic term in closed form, in place: s -> s' = bn (s - mean s) +
// b0 mean s (bn: B(k) for every k != 0, b0: B(0)), i.e. irfft(B rfft(s))
// exactly (elastic.py:250-263); the mean and the product in FP64, s' rounded
// once to FP32.  One block, a fixed summation order.
constexpr int kElastic1dThreads32 = 1024;
constexpr int64_t kElastic1dMax32 = 16384;
__global__ void __launch_bounds__(kElastic1dThreads32)
    k32_elastic1d(float *s, int64_t n, double bn, double b0, const unsigned *halt) {
  __shared__ double red[kElastic1dThreads32 / 32];
  pdl_wait();
  if (*halt) return;
  const int t = threadIdx.x;
  double acc = 0.0;
  for (int64_t i = t; i < n; i += kElastic1dThreads32) acc = acc + (double)s[i];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) acc = acc + __shfl_xor_sync(0xffffffffu, acc, o);
  if ((t & 31) == 0) red[t >> 5] = acc;
  __syncthreads();
  double tot = red[0];
  for (int w = 1; w < kElastic1dThreads32 / 32; ++w) tot = tot + red[w];
  const double mean = tot / (double)n;
  for (int64_t i = t; i < n; i += kElastic1dThreads32)
    s[i] = (float)(bn * ((double)s[i] - mean) + b0 * mean);
}

__global__ void k32_bmul(cufftComplex *__restrict__ k, const float *__restrict__ bk, int64_t nk,
                         const unsigned *halt) {
  if (halt && *halt) return;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nk;
       i += (int64_t)gridDim.x * blockDim.x) {
    const float b = bk[i];
    cufftComplex v = k[i];
    v.x *= b;
    v.y *= b;
    k[i] = v;
  }
}

// ------------------------------------------------------------------------
// Host side
// ------------------------------------------------------------------------
constexpr int kTX1_32 = 128;
constexpr int kGraphSteps32 = 50;

struct Variant32 {
  int tx, ty, minb;
  bool split;
  size_t smem2d, smem3d;
  void (*set_attrs)();
  void (*launch2d)(dim3, dim3, size_t, cudaStream_t, const Rate32 &);
  void (*launch3d)(dim3, dim3, size_t, cudaStream_t, const Rate32 &, int);
  std::string (*kernels)(int dim);     // the kernel instances of a 2D/3D rate stage
};

template <int TX, int TY, int MINB, bool WIN = true, int SORT = 0, bool PP = false>
Variant32 make_variant32() {
  Variant32 v;
  v.tx = TX;
  v.ty = TY;
  v.minb = MINB;
  v.split = false;
  v.smem2d = tile2d32_smem<TX, TY, SORT>();
  v.smem3d = march3d32_smem<TX, TY, SORT>();
  v.set_attrs = []() {
    const auto a = cudaFuncAttributeMaxDynamicSharedMemorySize;
    cudaFuncSetAttribute(k32_rate_tile2d<TX, TY, MINB, WIN, SORT, false, PP>, a,
                         (int)tile2d32_smem<TX, TY, SORT>());
    cudaFuncSetAttribute(k32_rate_march3d<TX, TY, MINB, WIN, SORT>, a,
                         (int)march3d32_smem<TX, TY, SORT>());
  };
  v.launch2d = [](dim3 g, dim3 b, size_t sm, cudaStream_t s, const Rate32 &P) {
    launch_pdl(k32_rate_tile2d<TX, TY, MINB, WIN, SORT, false, PP>, g, b, sm, s, P);
  };
  v.launch3d = [](dim3 g, dim3 b, size_t sm, cudaStream_t s, const Rate32 &P, int zc) {
    launch_pdl(k32_rate_march3d<TX, TY, MINB, WIN, SORT>, g, b, sm, s, P, zc);
  };
  v.kernels = [](int dim) {
    if (dim == 2) return kname("k32_rate_tile2d", {TX, TY, MINB, WIN, SORT, 0, PP});
    return kname("k32_rate_march3d", {TX, TY, MINB, WIN, SORT});
  };
  return v;
}

// Split variant: k32_chem (K points per work item, KMINB resident blocks)
// over all points, then the tile kernel (2D) or the marching flux kernel
// (3D, PP: per-point faces) reading mu/M back.
template <int TX, int TY, int MINB, int K, int KMINB, bool PP = false>
Variant32 make_split_variant32() {
  Variant32 v;
  v.tx = TX;
  v.ty = TY;
  v.minb = MINB;
  v.split = true;
  v.smem2d = tile2d32_smem<TX, TY>();
  v.smem3d = Flux3Geom<TX, TY>::smem(PP);
  v.set_attrs = []() {
    const auto a = cudaFuncAttributeMaxDynamicSharedMemorySize;
    cudaFuncSetAttribute(k32_rate_tile2d<TX, TY, MINB, false, false, true>, a,
                         (int)tile2d32_smem<TX, TY>());
    cudaFuncSetAttribute(k32_flux3<TX, TY, MINB, PP>, a, (int)Flux3Geom<TX, TY>::smem(PP));
    chem32_attrs<2, K, KMINB>();
    chem32_attrs<3, K, KMINB>();
  };
  v.launch2d = [](dim3 g, dim3 b, size_t sm, cudaStream_t s, const Rate32 &P) {
    launch_chem32<2, K, KMINB>(s, P);
    launch_pdl(k32_rate_tile2d<TX, TY, MINB, false, false, true>, g, b, sm, s, P);
  };
  v.launch3d = [](dim3 g, dim3 b, size_t sm, cudaStream_t s, const Rate32 &P, int zc) {
    launch_chem32<3, K, KMINB>(s, P);
    launch_pdl(k32_flux3<TX, TY, MINB, PP>, g, b, sm, s, P, zc);
  };
  v.kernels = [](int dim) {
    const std::string chem = kname("k32_chem", {dim, K, KMINB}) + " + ";
    if (dim == 2) return chem + kname("k32_rate_tile2d", {TX, TY, MINB, 0, 0, 1, 0});
    return chem + kname("k32_flux3", {TX, TY, MINB, PP});
  };
  return v;
}

const std::vector<Variant32> &variants32() {
  static const std::vector<Variant32> v = {
      make_variant32<32, 8, 2>(), make_variant32<32, 8, 3>(), make_variant32<32, 8, 4>(),
      make_variant32<32, 4, 6>(), make_variant32<64, 4, 3>(), make_variant32<32, 16, 2>(),
      make_variant32<32, 8, 2, false>(), make_variant32<32, 16, 2, false>(),
      make_variant32<32, 8, 2, true, true>(), make_variant32<32, 8, 3, false, true>(),
      make_variant32<32, 16, 2, false, true>(), make_variant32<32, 8, 2, false, true>(),
      make_variant32<32, 8, 3, false, true, true>(), make_variant32<32, 16, 2, false, true, true>(),
      make_variant32<32, 8, 3, false, 2, true>(), make_variant32<32, 16, 2, false, 2, true>(),
      make_variant32<32, 16, 2, false, 2, false>(),
      make_variant32<32, 8, 3, false, false, true>(), make_variant32<32, 16, 2, false, false, true>(),
      make_split_variant32<32, 8, 3, 2, 4, true>(), make_split_variant32<32, 8, 3, 4, 2, true>(),
      make_split_variant32<32, 8, 3, 2, 4, false>(), make_split_variant32<32, 8, 3, 4, 2, false>(),
      make_split_variant32<32, 16, 1, 4, 2, true>(), make_split_variant32<32, 4, 6, 4, 2, true>(),
      make_split_variant32<64, 4, 3, 4, 2, true>(), make_split_variant32<32, 8, 3, 2, 3, true>()};
  return v;
}

struct Stepper32 {
  pf5d_stepper_desc d{};
  bool closed1d = false;         // 1D elastic term in closed form (k32_elastic1d)
  ColPass2D colp;                // 2D elastic term: row transforms + one column kernel
  bool use_colpass = false;
  double bn = 0.0, b0 = 0.0;     // its B(k): bn for every k != 0, b0 at k = 0
  int64_t shape[3] = {1, 1, 1};
  int64_t npts = 0, nk = 0;
  float4 *hi = nullptr, *lo = nullptr, *dX = nullptr;
  float *s = nullptr, *bk = nullptr;
  cufftComplex *k = nullptr;
  cufftHandle fwd = 0, inv = 0;
  bool plans = false;
  double *mass_ws = nullptr;
  double *partial = nullptr;     // rate kernel block maxima
  float *mm = nullptr;           // split-rate buffers: mu, M, (M_Fe, X_Fe) per point
  StepState32 *st = nullptr;
  Rate32 rp{};
  Update32 up{};
  cudaStream_t cap = nullptr;
  std::map<int64_t, cudaGraphExec_t> graphs;
  dim3 grid, block;
  size_t smem = 0;
  int zc = 1;
  int variant = 0;
  std::string kernels;           // text returned by s32_rate_kernels
};

#define PF5D_CUFFT32(call)                                                         \
  do {                                                                             \
    cufftResult r_ = (call);                                                       \
    if (r_ != CUFFT_SUCCESS) {                                                     \
      set_error("%s:%d %s: cufft error %d", __FILE__, __LINE__, #call, (int)r_);   \
      return PF5D_ERR_CUFFT;                                                       \
    }                                                                              \
  } while (0)

// Grid of the rate kernel of `variant` (and the 3D axis-0 chunk).
static dim3 grid32_of(const Stepper32 *h, int variant, int *zc_out) {
  const Rate32 &P = h->rp;
  *zc_out = 1;
  if (h->d.dim == 1) return dim3((unsigned)((P.nx + kTX1_32 - 1) / kTX1_32));
  const Variant32 &v = variants32()[variant];
  const unsigned gx = (unsigned)((P.nx + v.tx - 1) / v.tx), gy = (unsigned)((P.ny + v.ty - 1) / v.ty);
  if (h->d.dim == 2) return dim3(gx, gy, 1);
  const int64_t tiles = (int64_t)gx * gy;
  const int64_t target = (int64_t)sm_count() * v.minb * 4;
  int64_t zc = (tiles * P.nz + target - 1) / target;
  zc = std::max<int64_t>(4, std::min<int64_t>(zc, 64));
  zc = std::min<int64_t>(zc, P.nz);
  *zc_out = (int)zc;
  return dim3(gx, gy, (unsigned)((P.nz + zc - 1) / zc));
}

// Block slots needed by the largest rate grid over all variants.
static int64_t max_blocks32(const Stepper32 *h) {
  int64_t m = 1;
  const int nv = h->d.dim == 1 ? 1 : (int)variants32().size();
  for (int v = 0; v < nv; ++v) {
    int zc = 1;
    const dim3 g = grid32_of(h, v, &zc);
    m = std::max<int64_t>(m, (int64_t)g.x * g.y * g.z);
  }
  return m;
}

static pf5d_status configure32(Stepper32 *h, int variant) {
  if (h->d.dim == 1) {
    h->block = dim3(kTX1_32);
    h->grid = grid32_of(h, 0, &h->zc);
    h->smem = 0;
    return PF5D_OK;
  }
  const auto &vars = variants32();
  PF5D_REQUIRE(variant >= 0 && variant < (int)vars.size(), PF5D_ERR_ARG, "bad variant %d",
               variant);
  const Variant32 &v = vars[variant];
  h->variant = variant;
  v.set_attrs();
  PF5D_LAUNCHED();
  h->block = dim3(v.tx, v.ty);
  h->smem = h->d.dim == 2 ? v.smem2d : v.smem3d;
  h->grid = grid32_of(h, variant, &h->zc);
  return PF5D_OK;
}

static pf5d_status launch_rate32(Stepper32 *h, cudaStream_t s) {
  switch (h->d.dim) {
    case 1: launch_pdl(k32_rate_1d<kTX1_32>, h->grid, h->block, 0, s, h->rp); break;
    case 2: variants32()[h->variant].launch2d(h->grid, h->block, h->smem, s, h->rp); break;
    default: variants32()[h->variant].launch3d(h->grid, h->block, h->smem, s, h->rp, h->zc);
  }
  PF5D_LAUNCHED();
  PF5D_CUDA(launch_pdl(k32_dt, dim3(1), dim3(kDt32Threads), 0, s, h->rp,
                       (int)(h->grid.x * h->grid.y * h->grid.z)));
  return PF5D_OK;
}

// The elastic term of a step: s -> s' in place, by cuFFT R2C, the B(k)/N
// multiply and C2R, or in 1D by k32_elastic1d (the closed form).
static pf5d_status elastic32(Stepper32 *h, cudaStream_t s) {
  if (h->closed1d) {
    PF5D_CUDA(launch_pdl(k32_elastic1d, dim3(1), dim3(kElastic1dThreads32), 0, s, h->s, h->npts,
                         h->bn, h->b0, (const unsigned *)&h->st->halt));
    return PF5D_OK;
  }
  if (h->use_colpass) {
    pf5d_status st;
    if ((st = colpass_rows_forward32(&h->colp, h->s, h->k, s)) != PF5D_OK) return st;
    if ((st = colpass_columns32(&h->colp, h->k, h->bk, &h->st->halt, s)) != PF5D_OK) return st;
    return colpass_rows_inverse32(&h->colp, h->k, h->s, s);
  }
    PF5D_CUFFT32(cufftSetStream(h->fwd, s));
    PF5D_CUFFT32(cufftExecR2C(h->fwd, h->s, h->k));
    k32_bmul<<<grid_for(h->nk, 256), 256, 0, s>>>(h->k, h->bk, h->nk, &h->st->halt);
    PF5D_LAUNCHED();
    PF5D_CUFFT32(cufftSetStream(h->inv, s));
    PF5D_CUFFT32(cufftExecC2R(h->inv, h->k, h->s));
  return PF5D_OK;
}

static pf5d_status enqueue32(Stepper32 *h, cudaStream_t s) {
  if (h->d.elastic) {
    const pf5d_status e = elastic32(h, s);
    if (e != PF5D_OK) return e;
  }
  pf5d_status st = launch_rate32(h, s);
  if (st != PF5D_OK) return st;
  PF5D_CUDA(launch_pdl(k32_update, dim3(grid_for(h->npts, 256, 4)), dim3(256), 0, s, h->up));
  PF5D_LAUNCHED();
  return PF5D_OK;
}

static pf5d_status graph32(Stepper32 *h, int64_t n, cudaGraphExec_t *out) {
  auto it = h->graphs.find(n);
  if (it != h->graphs.end()) {
    *out = it->second;
    return PF5D_OK;
  }
  cudaGraph_t g = nullptr;
  PF5D_CUDA(cudaStreamBeginCapture(h->cap, cudaStreamCaptureModeThreadLocal));
  pf5d_status st = PF5D_OK;
  for (int64_t i = 0; i < n && st == PF5D_OK; ++i) st = enqueue32(h, h->cap);
  cudaError_t e = cudaStreamEndCapture(h->cap, &g);
  if (st != PF5D_OK) {
    if (g) cudaGraphDestroy(g);
    return st;
  }
  PF5D_REQUIRE(e == cudaSuccess, PF5D_ERR_CUDA, "graph capture: %s", cudaGetErrorString(e));
  cudaGraphExec_t exec = nullptr;
  e = cudaGraphInstantiate(&exec, g, 0);
  cudaGraphDestroy(g);
  PF5D_REQUIRE(e == cudaSuccess, PF5D_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(e));
  h->graphs[n] = exec;
  *out = exec;
  return PF5D_OK;
}

static void drop_graphs(Stepper32 *h) {
  for (auto &kv : h->graphs) cudaGraphExecDestroy(kv.second);
  h->graphs.clear();
}

pf5d_status s32_create(const pf5d_stepper_desc *desc, const double *X_init, void *stream,
                       Stepper32 **out) {
  PF5D_REQUIRE(desc && X_init && out && desc->grid32, PF5D_ERR_ARG, "null argument");
  PF5D_REQUIRE(desc->node_stride32 == kStride32 && (((uintptr_t)desc->grid32) & 15) == 0,
               PF5D_ERR_ARG, "FP32 table needs %d floats per node, 16-byte aligned", kStride32);
  auto *h = new Stepper32();
  h->d = *desc;
  h->d.bk = nullptr;
  int64_t npts = 1;
  for (int d = 0; d < desc->dim; ++d) {
    h->shape[d] = desc->shape[d];
    npts *= desc->shape[d];
  }
  h->npts = npts;
  auto fail = [&](pf5d_status code) {
    s32_destroy(h);
    return code;
  };
  if (cudaMalloc(&h->hi, npts * sizeof(float4)) != cudaSuccess ||
      cudaMalloc(&h->lo, npts * sizeof(float4)) != cudaSuccess ||
      cudaMalloc(&h->dX, npts * sizeof(float4)) != cudaSuccess ||
      cudaMalloc(&h->st, sizeof(StepState32)) != cudaSuccess ||
      cudaMalloc(&h->mass_ws, (kMassBlocks * S + S) * sizeof(double)) != cudaSuccess ||
      cudaStreamCreateWithFlags(&h->cap, cudaStreamNonBlocking) != cudaSuccess) {
    set_error("device allocation failed");
    return fail(PF5D_ERR_CUDA);
  }
  if (desc->elastic) {
    long long n[3];
    for (int d = 0; d < desc->dim; ++d) n[d] = desc->shape[d];
    h->nk = npts / desc->shape[desc->dim - 1] * (desc->shape[desc->dim - 1] / 2 + 1);
    size_t ws = 0;
    if (cufftCreate(&h->fwd) != CUFFT_SUCCESS || cufftCreate(&h->inv) != CUFFT_SUCCESS ||
        cufftMakePlanMany64(h->fwd, desc->dim, n, nullptr, 1, 0, nullptr, 1, 0, CUFFT_R2C, 1,
                            &ws) != CUFFT_SUCCESS ||
        cufftMakePlanMany64(h->inv, desc->dim, n, nullptr, 1, 0, nullptr, 1, 0, CUFFT_C2R, 1,
                            &ws) != CUFFT_SUCCESS) {
      set_error("cuFFT plan creation failed");
      return fail(PF5D_ERR_CUFFT);
    }
    h->plans = true;
    if (desc->dim == 1 && npts <= kElastic1dMax32) {
      // 1D B(k) is one value for every k != 0 (checked exactly): closed form
      bool flat = true;
      for (int64_t i = 2; i < h->nk && flat; ++i) flat = desc->bk[i] == desc->bk[1];
      h->closed1d = flat;
      h->bn = h->nk > 1 ? desc->bk[1] : 0.0;
      h->b0 = desc->bk[0];
    }
    std::vector<float> b(h->nk);
    const double inv_n = 1.0 / (double)npts;
    for (int64_t i = 0; i < h->nk; ++i) b[i] = (float)(desc->bk[i] * inv_n);
    if (cudaMalloc(&h->s, npts * sizeof(float)) != cudaSuccess ||
        cudaMalloc(&h->k, h->nk * sizeof(cufftComplex)) != cudaSuccess ||
        cudaMalloc(&h->bk, h->nk * sizeof(float)) != cudaSuccess ||
        cudaMemcpy(h->bk, b.data(), h->nk * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess) {
      set_error("device allocation failed");
      return fail(PF5D_ERR_CUDA);
    }
    const int64_t n0 = h->shape[0];
    if (desc->dim == 2 && n0 >= 8 && n0 <= 1024 && (n0 & (n0 - 1)) == 0) {
      h->use_colpass = colpass_create(h->shape, &h->colp, true) == PF5D_OK;
      if (!h->use_colpass) colpass_destroy(&h->colp);
    }
  }
  Rate32 &P = h->rp;
  if (desc->dim == 1) {
    P.nz = 1; P.ny = 1; P.nx = (int)h->shape[0];
  } else if (desc->dim == 2) {
    P.nz = 1; P.ny = (int)h->shape[0]; P.nx = (int)h->shape[1];
  } else {
    P.nz = (int)h->shape[0]; P.ny = (int)h->shape[1]; P.nx = (int)h->shape[2];
  }
  P.D = h->hi;
  P.sp = desc->elastic ? h->s : nullptr;
  P.dX = h->dX;
  Table32 &T = P.T;
  T.grid = desc->grid32;
  T.coord = desc->node_coord;
  T.n = desc->table_n;
  T.stride = kStride32;
  T.inv_step = 1.0 / desc->resolution;
  T.inv_step_f = (float)T.inv_step;
  T.threshold = 1.0 - 4.0 * desc->resolution - 1e-9;
  T.max_nn_dist = desc->max_nn_dist;
  double sx = 0.0;
  for (int c = 0; c < S; ++c) {
    const double u = desc->x0[c] * T.inv_step;
    const double fl = floor(u);
    T.ib[c] = (int)fl;
    T.fb[c] = (float)(u - fl);
    T.x0[c] = desc->x0[c];
    sx = sx + desc->x0[c];
    P.kappa[c] = (float)desc->kappa[c];
    P.lvec[c] = (float)desc->lvec[c];
    P.x0f[c] = (float)desc->x0[c];
  }
  T.sum_x0 = sx;
  P.c_fe = 1.0 - sx;
  P.flux_scale = (float)(0.5 / (desc->dx * desc->dx));
  P.inv_dx2 = (float)(1.0 / (desc->dx * desc->dx));
  P.ctld = desc->ctld;
  P.t_cfl = desc->t_cfl;
  P.lower = desc->lower_limit;
  P.upper = desc->upper_limit;
  P.factor = desc->max_change_factor;
  P.adaptive = desc->adaptive;
  P.st = h->st;
  if (cudaMalloc(&h->partial, (size_t)max_blocks32(h) * sizeof(double)) != cudaSuccess) {
    set_error("device allocation failed");
    return fail(PF5D_ERR_CUDA);
  }
  P.partial = h->partial;
  P.npts = npts;
  // split buffers: mu (float4), M (float4), (M_Fe, X_Fe) (float2) per point
  if (cudaMalloc(&h->mm, (size_t)npts * (2 * sizeof(float4) + sizeof(float2))) != cudaSuccess) {
    set_error("device allocation failed");
    return fail(PF5D_ERR_CUDA);
  }
  P.mm_mu = reinterpret_cast<float4 *>(h->mm);
  P.mm_m = P.mm_mu + npts;
  P.mm_f = reinterpret_cast<float2 *>(P.mm_m + npts);
  Update32 &U = h->up;
  U.hi = h->hi;
  U.lo = h->lo;
  U.dX = h->dX;
  U.npts = npts;
  U.st = h->st;
  for (int c = 0; c < S; ++c) {
    U.x0[c] = desc->x0[c];
    U.lvec[c] = (float)desc->lvec[c];
  }
  U.sum_x0 = sx;
  U.s = desc->elastic ? h->s : nullptr;
  U.oob_interval = desc->oob_interval;
  pf5d_status st = configure32(h, 0);
  if (st != PF5D_OK) return fail(st);
  if ((st = s32_reset(h, X_init, desc->dt0, 0.0, stream)) != PF5D_OK) return fail(st);
  *out = h;
  return PF5D_OK;
}

pf5d_status s32_reset(Stepper32 *h, const double *X, double dt, double time, void *stream) {
  cudaStream_t s = as_stream(stream);
  StepState32 init{};
  init.dt = dt;
  init.time = time;
  PF5D_CUDA(cudaMemcpyAsync(h->st, &init, sizeof(init), cudaMemcpyHostToDevice, s));
  if (X) {
    k32_split<<<grid_for(h->npts, 256, 4), 256, 0, s>>>(X, h->npts, h->up);
    PF5D_LAUNCHED();
  }
  PF5D_CUDA(cudaStreamSynchronize(s));
  return PF5D_OK;
}

pf5d_status s32_advance(Stepper32 *h, int64_t nsteps, void *stream) {
  cudaStream_t s = as_stream(stream);
  while (nsteps > 0) {
    const int64_t n = nsteps < kGraphSteps32 ? nsteps : kGraphSteps32;
    cudaGraphExec_t g = nullptr;
    pf5d_status st = graph32(h, n, &g);
    if (st != PF5D_OK) return st;
    PF5D_CUDA(cudaGraphLaunch(g, s));
    nsteps -= n;
  }
  return PF5D_OK;
}

pf5d_status s32_state(Stepper32 *h, pf5d_step_state *out, void *stream) {
  StepState32 hs;
  cudaStream_t s = as_stream(stream);
  PF5D_CUDA(cudaMemcpyAsync(&hs, h->st, sizeof(hs), cudaMemcpyDeviceToHost, s));
  PF5D_CUDA(cudaStreamSynchronize(s));
  out->dt = hs.dt;
  out->time = hs.time;
  out->xdotmax = hs.xdotmax;
  out->step = hs.step;
  out->flags = hs.flags | (hs.halt ? PF5D_FLAG_HALTED : 0u);
  out->halted = hs.halt;
  return PF5D_OK;
}

// FP64 copies for the save-step reductions: dX/dt (4 per point) and mu/M
// (SoA, 9 rows), from the FP32 buffers.
__global__ void k32_widen(const float *__restrict__ src, int64_t n, double *__restrict__ dst) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    dst[i] = (double)src[i];
}

// FP64 mu/M rows (SoA, 9 rows: mu_1..4, M_Fe, M_1..4) from the split buffers.
__global__ void k32_widen_mm(Rate32 P, double *__restrict__ dst) {
  const int64_t n = P.npts;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const float4 mu = P.mm_mu[i], m = P.mm_m[i];
    const float2 f = P.mm_f[i];
    const float v[NP] = {mu.x, mu.y, mu.z, mu.w, f.x, m.x, m.y, m.z, m.w};
#pragma unroll
    for (int r = 0; r < NP; ++r) dst[r * n + i] = (double)v[r];
  }
}

pf5d_status s32_step_save_inputs(Stepper32 *h, double *X_out, double *dX_out, double *mm_out,
                                 void *stream) {
  cudaStream_t s = as_stream(stream);
  if (h->d.elastic) {
    const pf5d_status e = elastic32(h, s);
    if (e != PF5D_OK) return e;
  }
  pf5d_status st = launch_rate32(h, s);
  if (st != PF5D_OK) return st;
  switch (h->d.dim) {
    case 1: chem32_attrs<1, 2, 3>(); launch_chem32<1, 2, 3>(s, h->rp); break;
    case 2: chem32_attrs<2, 2, 3>(); launch_chem32<2, 2, 3>(s, h->rp); break;
    default: chem32_attrs<3, 2, 3>(); launch_chem32<3, 2, 3>(s, h->rp);
  }
  PF5D_LAUNCHED();
  k32_join<<<grid_for(h->npts, 256, 4), 256, 0, s>>>(h->hi, h->lo, h->npts, h->up, X_out);
  PF5D_LAUNCHED();
  k32_widen<<<grid_for(4 * h->npts, 256, 4), 256, 0, s>>>(reinterpret_cast<const float *>(h->dX),
                                                          4 * h->npts, dX_out);
  PF5D_LAUNCHED();
  k32_widen_mm<<<grid_for(h->npts, 256, 4), 256, 0, s>>>(h->rp, mm_out);
  PF5D_LAUNCHED();
  return PF5D_OK;
}

pf5d_status s32_step_update(Stepper32 *h, void *stream) {
  cudaStream_t s = as_stream(stream);
  k32_update<<<grid_for(h->npts, 256, 4), 256, 0, s>>>(h->up);
  PF5D_LAUNCHED();
  return PF5D_OK;
}

pf5d_status s32_field(Stepper32 *h, double *X_out, void *stream) {
  cudaStream_t s = as_stream(stream);
  k32_join<<<grid_for(h->npts, 256, 4), 256, 0, s>>>(h->hi, h->lo, h->npts, h->up, X_out);
  PF5D_LAUNCHED();
  return PF5D_OK;
}

pf5d_status s32_mass(Stepper32 *h, double *mean_out, void *stream) {
  cudaStream_t s = as_stream(stream);
  const unsigned nb = std::min<unsigned>(kMassBlocks, grid_for(h->npts, 256, 4));
  k32_mass_partial<<<nb, 256, 0, s>>>(h->hi, h->lo, h->npts, h->mass_ws);
  PF5D_LAUNCHED();
  k32_mass_final<<<1, 32, 0, s>>>(h->mass_ws, (int)nb, h->mass_ws + kMassBlocks * S);
  PF5D_LAUNCHED();
  double sums[S];
  PF5D_CUDA(cudaMemcpyAsync(sums, h->mass_ws + kMassBlocks * S, sizeof(sums),
                            cudaMemcpyDeviceToHost, s));
  PF5D_CUDA(cudaStreamSynchronize(s));
  for (int c = 0; c < S; ++c) mean_out[c] = h->d.x0[c] + sums[c] / (double)h->npts;
  return PF5D_OK;
}

int32_t s32_variant_count() { return (int32_t)variants32().size(); }

const char *s32_rate_kernels(Stepper32 *h) {
  if (h->d.dim == 1) h->kernels = kname("k32_rate_1d", {kTX1_32});
  else h->kernels = variants32()[h->variant].kernels(h->d.dim);
  h->kernels += " + k32_dt";
  return h->kernels.c_str();
}

int32_t s32_launches_per_step(const Stepper32 *h) {
  const bool split = h->d.dim >= 2 && variants32()[h->variant].split;
  return (split ? 4 : 3) + (h->d.elastic ? 1 : 0);   // rate (+chem), dt, update (+ B(k))
}

pf5d_status s32_set_variant(Stepper32 *h, int32_t variant) {
  pf5d_status st = configure32(h, variant);
  if (st == PF5D_OK) drop_graphs(h);
  return st;
}

pf5d_status s32_autotune(Stepper32 *h, int32_t *variant, float *best_ms, void *stream) {
  cudaStream_t s = as_stream(stream);
  if (h->d.dim == 1) {
    if (variant) *variant = 0;
    if (best_ms) *best_ms = 0.f;
    return PF5D_OK;
  }
  StepState32 saved;
  PF5D_CUDA(cudaMemcpyAsync(&saved, h->st, sizeof(saved), cudaMemcpyDeviceToHost, s));
  PF5D_CUDA(cudaStreamSynchronize(s));
  cudaEvent_t e0, e1;
  PF5D_CUDA(cudaEventCreate(&e0));
  PF5D_CUDA(cudaEventCreate(&e1));
  int best = h->variant;
  float best_t = 1e30f;
  for (int v = 0; v < (int)variants32().size(); ++v) {
    if (configure32(h, v) != PF5D_OK) continue;
    if (launch_rate32(h, s) != PF5D_OK) {
      cudaGetLastError();
      continue;
    }
    PF5D_CUDA(cudaEventRecord(e0, s));
    pf5d_status st = PF5D_OK;
    for (int r = 0; r < 5 && st == PF5D_OK; ++r) st = launch_rate32(h, s);
    PF5D_CUDA(cudaEventRecord(e1, s));
    PF5D_CUDA(cudaEventSynchronize(e1));
    float ms = 0.f;
    PF5D_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    if (st == PF5D_OK && ms / 5 < best_t) {
      best_t = ms / 5;
      best = v;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  pf5d_status st = configure32(h, best);
  if (st != PF5D_OK) return st;
  drop_graphs(h);
  PF5D_CUDA(cudaMemcpyAsync(h->st, &saved, sizeof(saved), cudaMemcpyHostToDevice, s));
  PF5D_CUDA(cudaStreamSynchronize(s));
  if (variant) *variant = best;
  if (best_ms) *best_ms = best_t;
  return PF5D_OK;
}

pf5d_status s32_launch_stage(Stepper32 *h, int32_t stage, void *stream) {
  cudaStream_t s = as_stream(stream);
  switch (stage) {
    case PF5D_STAGE_RATE:
      return launch_rate32(h, s);
    case PF5D_STAGE_UPDATE:
      k32_update<<<grid_for(h->npts, 256, 4), 256, 0, s>>>(h->up);
      PF5D_LAUNCHED();
      return PF5D_OK;
    // 1D closed form: the whole elastic term is the FFT_FWD stage
    case PF5D_STAGE_FFT_FWD:
      PF5D_REQUIRE(h->d.elastic, PF5D_ERR_ARG, "elasticity is off");
      if (h->closed1d) return elastic32(h, s);
      if (h->use_colpass) return colpass_rows_forward32(&h->colp, h->s, h->k, s);
      PF5D_CUFFT32(cufftSetStream(h->fwd, s));
      PF5D_CUFFT32(cufftExecR2C(h->fwd, h->s, h->k));
      return PF5D_OK;
    case PF5D_STAGE_BMUL:
      PF5D_REQUIRE(h->d.elastic, PF5D_ERR_ARG, "elasticity is off");
      if (h->closed1d) return PF5D_OK;
      if (h->use_colpass) return colpass_columns32(&h->colp, h->k, h->bk, &h->st->halt, s);
      k32_bmul<<<grid_for(h->nk, 256), 256, 0, s>>>(h->k, h->bk, h->nk, &h->st->halt);
      PF5D_LAUNCHED();
      return PF5D_OK;
    case PF5D_STAGE_FFT_INV:
      PF5D_REQUIRE(h->d.elastic, PF5D_ERR_ARG, "elasticity is off");
      if (h->closed1d) return PF5D_OK;
      if (h->use_colpass) return colpass_rows_inverse32(&h->colp, h->k, h->s, s);
      PF5D_CUFFT32(cufftSetStream(h->inv, s));
      PF5D_CUFFT32(cufftExecC2R(h->inv, h->k, h->s));
      return PF5D_OK;
    default:
      set_error("unknown stage %d", stage);
      return PF5D_ERR_ARG;
  }
}

float *s32_rate(Stepper32 *h) { return reinterpret_cast<float *>(h->dX); }

void s32_destroy(Stepper32 *h) {
  if (!h) return;
  drop_graphs(h);
  if (h->plans) {
    cufftDestroy(h->fwd);
    cufftDestroy(h->inv);
  }
  cudaFree(h->hi);
  cudaFree(h->lo);
  cudaFree(h->dX);
  cudaFree(h->s);
  cudaFree(h->bk);
  colpass_destroy(&h->colp);
  cudaFree(h->k);
  cudaFree(h->st);
  cudaFree(h->mass_ws);
  cudaFree(h->partial);
  cudaFree(h->mm);
  if (h->cap) cudaStreamDestroy(h->cap);
  delete h;
}

}  // namespace pf5d
