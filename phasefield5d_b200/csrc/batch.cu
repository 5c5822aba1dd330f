// batch.cu -- many independent solves advanced together (the batched form).
//
// Solves of different dimension (1D / 2D), size, composition, temperature
// table and kappa are split into two lanes (balanced by points); the solves
// of a lane share every launch of its step:
//   * one cuFFT R2C/C2R pair per group of 2D solves with the same shape
//     (batched plans; B(k) depends only on the direction of k, so a shape
//     group shares one B(k)/N) and its B(k) multiply, the groups' chains on
//     parallel graph branches;
//   * one persistent rate launch: blocks loop over the lane's tiles
//     (32x8-style plane tiles for 2D, runs of TX*TY points for 1D) and
//     store each tile's max|dX/dt| in its own slot;
//   * kb_dt: one warp per solve reduces its slots and runs its FP64 dt
//     controller;
//   * one persistent compensated-update launch over fixed 1024-point chunks.
// The two lanes' chains are separate branches of the step graph, the second
// one FFT phase behind, so one lane's FFTs run beside the other's rate kernel.
// In 1D, B(k) is the same constant B_n for every k != 0 and zero at k = 0,
// so the elastic term is exactly B_n * (s - mean(s)): 1D solves need no FFT.
// The mean (the k = 0 mode) is formed in FP64 from per-chunk partial sums
// in a fixed order.  Every per-solve reduction has a fixed order, so a
// solve's trajectory does not depend on which other solves share the batch.
#include <algorithm>
#include <map>
#include <vector>

#include <cufft.h>

#include "pf5d_fp32c.cuh"
#include "pf5d_host.h"

namespace pf5d {

constexpr int kChunk = 1024;              // points per update chunk
constexpr int kUpdThreads = 256;

struct BSolve {
  Rate32 R;            // per-solve rate parameters (R.D = hi, R.dX, R.sp, R.st, R.T, ...)
  int dim;             // 1 or 2
  int ntx, nty;        // tile grid
  int tile0, ntiles;   // global tile range
  int chunk0, nchunks; // global update-chunk range
  int emode;           // 0: elasticity off, 1: 1D constant-B form, 2: 2D cuFFT
  int oob_interval;
  int64_t npts;
  float4 *hi, *lo;
  float *s;            // misfit (update writes; 2D: FFT in/out, then s')
  double *spart;       // 1D: per-chunk FP64 partial sums of s
  float bn;            // 1D: B(k) for k != 0
  float lvec[S];
  double x0[S];
  double sum_x0;
};

// Largest i with key(i) <= t over a sorted prefix array inside the solves.
__device__ __forceinline__ int find_solve_tile(const BSolve *solves, int n, int t) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (solves[mid].tile0 <= t) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}
__device__ __forceinline__ int find_solve_chunk(const BSolve *solves, int n, int c) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (solves[mid].chunk0 <= c) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// One 1D tile: NT consecutive points of solve B (Rate32 copy in shared memory).
template <int NT>
__device__ __forceinline__ float tile1d32_body(const BSolve &B, const Rate32 &P, int tile,
                                               float *smf, unsigned *flags, int tid) {
  constexpr int HX = NT + 4, MX = NT + 2;
  float *Xs = smf;                 // [S][HX]
  float *Ms = Xs + S * HX;         // [NPM][MX]
  float *Fx = Ms + NPM * MX;       // [S][NT+1]
  const int x0 = tile * NT;
  const int n = P.nx;
  for (int pos = tid; pos < HX; pos += NT) {
    const float4 v = __ldg(P.D + wrap_any(x0 + pos - 2, n));
    Xs[0 * HX + pos] = v.x;
    Xs[1 * HX + pos] = v.y;
    Xs[2 * HX + pos] = v.z;
    Xs[3 * HX + pos] = v.w;
  }
  double mean = 0.0;
  if (B.emode == 1) {
    double acc = 0.0;
    for (int c = 0; c < B.nchunks; ++c) acc += B.spart[c];
    mean = acc / (double)n;
  }
  __syncthreads();
  for (int pos = tid; pos < MX; pos += NT) {
    const int px = pos + 1;
    float d[S], lap[S];
#pragma unroll
    for (int c = 0; c < S; ++c) {
      d[c] = Xs[c * HX + px];
      const float nb[2] = {Xs[c * HX + px + 1], Xs[c * HX + px - 1]};
      lap[c] = lap32<2>(nb, d[c], P.inv_dx2);
    }
    float spv = 0.f;
    if (B.emode == 1)
      spv = (float)((double)B.bn * ((double)__ldg(B.s + wrap_any(x0 + pos - 1, n)) - mean));
    float v[NPM];
    chem32(P, d, lap, spv, nullptr, nullptr, v, flags);
#pragma unroll
    for (int r = 0; r < NPM; ++r) Ms[r * MX + pos] = v[r];
  }
  __syncthreads();
  for (int f = tid; f < NT + 1; f += NT) {
    float J[S];
    face32_between<HX, MX>(P, Xs, Ms, f + 1, f, Xs, Ms, f + 2, f + 1, J);
#pragma unroll
    for (int c = 0; c < S; ++c) Fx[c * (NT + 1) + f] = J[c];
  }
  __syncthreads();
  float vmax = 0.f;
  if (x0 + tid < n) {
    float out[S];
#pragma unroll
    for (int c = 0; c < S; ++c)
      out[c] = (Fx[c * (NT + 1) + tid + 1] - Fx[c * (NT + 1) + tid]) * P.flux_scale;
    store_rate(P.dX, x0 + tid, out, vmax);
  }
  return vmax;
}

template <int TX, int TY, int SORT = 0>
struct BatchSmem {
  static constexpr int NT = TX * TY;
  static constexpr size_t s1d = (S * (NT + 4) + NPM * (NT + 2) + S * (NT + 1)) * sizeof(float);
  static constexpr size_t s2d = Tile2dSmem32<TX, TY, SORT>::bytes;
  // Rate32 copy, rounded up to whole float4 plus one spare float4, then the tile work area.
  static constexpr size_t head = 16 * ((sizeof(Rate32) + 15) / 16 + 1);
  static constexpr size_t rate = head + (s2d > s1d ? s2d : s1d);
};

template <int TX, int TY, int MINB, bool WIN, int SORT = 0, bool PP = false>
__global__ void __launch_bounds__(TX * TY, MINB)
    kb_rate(const BSolve *__restrict__ solves, int nsolves, int tile_begin, int tile_end,
            double *tile_max) {
  constexpr int NT = TX * TY;
  extern __shared__ float4 sm4[];
  Rate32 *Rs = reinterpret_cast<Rate32 *>(sm4);
  float4 *work = sm4 + BatchSmem<TX, TY, SORT>::head / 16;
  const int tid = threadIdx.y * TX + threadIdx.x;
  pdl_wait();
  for (int t = tile_begin + blockIdx.x; t < tile_end; t += gridDim.x) {
    const int si = find_solve_tile(solves, nsolves, t);
    const BSolve &B = solves[si];
    __syncthreads();                               // previous tile done with shared memory
    {
      const int *src = reinterpret_cast<const int *>(&B.R);
      int *dst = reinterpret_cast<int *>(Rs);
      for (int i = tid; i < (int)(sizeof(Rate32) / sizeof(int)); i += NT) dst[i] = src[i];
    }
    __syncthreads();
    const Rate32 &P = *Rs;
    if (P.st->halt) continue;
    const int local = t - B.tile0;
    unsigned flags = 0;
    float vmax;
    if (B.dim == 2)
      vmax = tile2d32_body<TX, TY, WIN, SORT, false, PP>(P, local % B.ntx, local / B.ntx, work,
                                                          &flags, tid);
    else
      vmax = tile1d32_body<NT>(B, P, local, reinterpret_cast<float *>(work), &flags, tid);
    raise_rate_flags(P.st, flags);
    double *red = reinterpret_cast<double *>(work);    // free after the body's last barrier
    __syncthreads();
    finish_slot32(vmax, red, tile_max + t);
  }
}

__global__ void __launch_bounds__(kUpdThreads)
    kb_update(const BSolve *__restrict__ solves, int nsolves, int chunk_begin, int chunk_end) {
  __shared__ double red[kUpdThreads / 32];
  const int tid = threadIdx.x;
  pdl_wait();
  for (int cidx = chunk_begin + blockIdx.x; cidx < chunk_end; cidx += gridDim.x) {
    const BSolve &B = solves[find_solve_chunk(solves, nsolves, cidx)];
    StepState32 *st = B.R.st;
    if (st->halt) continue;
    const int local = cidx - B.chunk0;
    const float dtf = (float)st->dt;
    const bool check = B.oob_interval > 0 && (st->step % B.oob_interval) == 0;
    unsigned f = 0;
    double ssum = 0.0;
    for (int k = 0; k < kChunk / kUpdThreads; ++k) {
      const int64_t p = (int64_t)local * kChunk + k * kUpdThreads + tid;
      if (p >= B.npts) break;
      const float4 H = B.hi[p], L = B.lo[p], Rr = B.R.dX[p];
      float h[S] = {H.x, H.y, H.z, H.w}, l[S] = {L.x, L.y, L.z, L.w};
      const float r[S] = {Rr.x, Rr.y, Rr.z, Rr.w};
#pragma unroll
      for (int c = 0; c < S; ++c) comp_add(h[c], l[c], __fmul_rn(dtf, r[c]));
      double dd[S], dsum = 0.0;
#pragma unroll
      for (int c = 0; c < S; ++c) {
        dd[c] = (double)h[c] + (double)l[c];
        dsum = dsum + dd[c];
      }
      const double total = B.sum_x0 + dsum;
      if (total > 1.0) {
        const double inv = 1.0 / total;
#pragma unroll
        for (int c = 0; c < S; ++c) {
          const double dn = (B.x0[c] + dd[c]) * inv - B.x0[c];
          h[c] = (float)dn;
          l[c] = (float)(dn - (double)h[c]);
          dd[c] = (double)h[c] + (double)l[c];
        }
      }
      B.hi[p] = make_float4(h[0], h[1], h[2], h[3]);
      B.lo[p] = make_float4(l[0], l[1], l[2], l[3]);
      if (B.emode) {
        float acc = 0.f;
#pragma unroll
        for (int c = 0; c < S; ++c) acc = fmaf(h[c] + l[c], B.lvec[c], acc);
        B.s[p] = acc;
        ssum += (double)acc;
      }
      if (check) {
        double x[S];
#pragma unroll
        for (int c = 0; c < S; ++c) x[c] = B.x0[c] + dd[c];
        f |= oob_flags_x(x);
      }
    }
    if (B.emode == 1) {                    // fixed-order FP64 chunk sum (k = 0 mode)
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) ssum += __shfl_xor_sync(0xffffffffu, ssum, o);
      __syncthreads();
      if ((tid & 31) == 0) red[tid >> 5] = ssum;
      __syncthreads();
      if (tid == 0) {
        double v = 0.0;
        for (int w = 0; w < kUpdThreads / 32; ++w) v += red[w];
        B.spart[local] = v;
      }
    }
    raise32(st, f);
  }
}

// Initial state of one solve: X (FP64 device) -> hi/lo, misfit, partial sums, OOB test.
__global__ void kb_split(const double *__restrict__ X, const BSolve *__restrict__ solves, int si) {
  __shared__ double red[kUpdThreads / 32];
  const BSolve &B = solves[si];
  const int tid = threadIdx.x;
  for (int chunk = blockIdx.x; chunk < B.nchunks; chunk += gridDim.x) {
    unsigned f = 0;
    double ssum = 0.0;
    for (int k = 0; k < kChunk / kUpdThreads; ++k) {
      const int64_t p = (int64_t)chunk * kChunk + k * kUpdThreads + tid;
      if (p >= B.npts) break;
      float h[S], l[S];
      double x[S];
#pragma unroll
      for (int c = 0; c < S; ++c) {
        x[c] = X[4 * p + c];
        const double d = x[c] - B.x0[c];
        h[c] = (float)d;
        l[c] = (float)(d - (double)h[c]);
      }
      B.hi[p] = make_float4(h[0], h[1], h[2], h[3]);
      B.lo[p] = make_float4(l[0], l[1], l[2], l[3]);
      if (B.emode) {
        float acc = 0.f;
#pragma unroll
        for (int c = 0; c < S; ++c) acc = fmaf(h[c] + l[c], B.lvec[c], acc);
        B.s[p] = acc;
        ssum += (double)acc;
      }
      if (B.oob_interval > 0) f |= oob_flags_x(x);
    }
    if (B.emode == 1) {
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) ssum += __shfl_xor_sync(0xffffffffu, ssum, o);
      __syncthreads();
      if ((tid & 31) == 0) red[tid >> 5] = ssum;
      __syncthreads();
      if (tid == 0) {
        double v = 0.0;
        for (int w = 0; w < kUpdThreads / 32; ++w) v += red[w];
        B.spart[chunk] = v;
      }
    }
    raise32(B.R.st, f);
  }
}

// Exact resume of one solve from its FP32 pair: copy hi/lo, recompute the
// misfit and the 1D partial sums exactly as the update kernel forms them.
__global__ void kb_resume(const float4 *__restrict__ hi_in, const float4 *__restrict__ lo_in,
                          const BSolve *__restrict__ solves, int si) {
  __shared__ double red[kUpdThreads / 32];
  const BSolve &B = solves[si];
  const int tid = threadIdx.x;
  for (int chunk = blockIdx.x; chunk < B.nchunks; chunk += gridDim.x) {
    double ssum = 0.0;
    for (int k = 0; k < kChunk / kUpdThreads; ++k) {
      const int64_t p = (int64_t)chunk * kChunk + k * kUpdThreads + tid;
      if (p >= B.npts) break;
      const float4 H = hi_in[p], L = lo_in[p];
      B.hi[p] = H;
      B.lo[p] = L;
      if (B.emode) {
        const float h[S] = {H.x, H.y, H.z, H.w}, l[S] = {L.x, L.y, L.z, L.w};
        float acc = 0.f;
#pragma unroll
        for (int c = 0; c < S; ++c) acc = fmaf(h[c] + l[c], B.lvec[c], acc);
        B.s[p] = acc;
        ssum += (double)acc;
      }
    }
    if (B.emode == 1) {
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) ssum += __shfl_xor_sync(0xffffffffu, ssum, o);
      __syncthreads();
      if ((tid & 31) == 0) red[tid >> 5] = ssum;
      __syncthreads();
      if (tid == 0) {
        double v = 0.0;
        for (int w = 0; w < kUpdThreads / 32; ++w) v += red[w];
        B.spart[chunk] = v;
      }
    }
  }
}

__global__ void kb_join(const BSolve *__restrict__ solves, int si, double *__restrict__ X) {
  const BSolve &B = solves[si];
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < B.npts;
       p += (int64_t)gridDim.x * blockDim.x) {
    const float4 H = B.hi[p], L = B.lo[p];
    const float h[S] = {H.x, H.y, H.z, H.w}, l[S] = {L.x, L.y, L.z, L.w};
#pragma unroll
    for (int c = 0; c < S; ++c) X[4 * p + c] = B.x0[c] + ((double)h[c] + (double)l[c]);
  }
}

// B(k)/N multiply over the spectra of one shape group (count solves, nk each).
__global__ void kb_bmul(cufftComplex *__restrict__ k, const float *__restrict__ bk, int64_t nk,
                        int64_t total) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total;
       i += (int64_t)gridDim.x * blockDim.x) {
    const float b = bk[i % nk];
    cufftComplex v = k[i];
    v.x *= b;
    v.y *= b;
    k[i] = v;
  }
}

// ------------------------------------------------------------------------
// Host side
// ------------------------------------------------------------------------
// The dt controllers of all solves after a rate launch: one warp per solve
// reduces its tiles' maxima and advances its dt / time / step.
__global__ void kb_dt(const BSolve *__restrict__ solves, int nsolves, const double *tile_max) {
  pdl_wait();
  const int i = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (i >= nsolves) return;
  const BSolve &B = solves[i];
  if (B.R.st->halt) return;
  dt_from_slots32(B.R, tile_max + B.tile0, B.ntiles);
}

struct BatchVariant {
  int tx, ty, minb;
  bool win;
  size_t smem;
  void (*set_attrs)();
  void (*launch)(int grid, cudaStream_t s, const BSolve *solves, int n, int tile_begin,
                 int tile_end, double *tile_max);
  int (*occupancy)();
};

template <int TX, int TY, int MINB, bool WIN, int SORT = 0, bool PP = false>
BatchVariant make_bvariant() {
  using SM = BatchSmem<TX, TY, SORT>;
  BatchVariant v;
  v.tx = TX;
  v.ty = TY;
  v.minb = MINB;
  v.win = WIN;
  v.smem = SM::rate;
  v.set_attrs = []() {
    cudaFuncSetAttribute(kb_rate<TX, TY, MINB, WIN, SORT, PP>,
                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SM::rate);
  };
  v.launch = [](int grid, cudaStream_t s, const BSolve *solves, int n, int tile_begin,
                int tile_end, double *tile_max) {
    launch_pdl(kb_rate<TX, TY, MINB, WIN, SORT, PP>, dim3(grid), dim3(TX, TY), SM::rate, s, solves, n,
               tile_begin, tile_end, tile_max);
  };
  v.occupancy = []() {
    int nb = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kb_rate<TX, TY, MINB, WIN, SORT, PP>, TX * TY,
                                                  SM::rate);
    return nb;
  };
  return v;
}

const std::vector<BatchVariant> &batch_variants() {
  static const std::vector<BatchVariant> v = {
      make_bvariant<32, 8, 2, true>(), make_bvariant<32, 8, 3, true>(),
      make_bvariant<32, 8, 2, false>(), make_bvariant<32, 8, 3, false>(),
      make_bvariant<32, 4, 4, true>(), make_bvariant<64, 4, 2, true>(),
      make_bvariant<32, 8, 2, false, true>(), make_bvariant<32, 8, 3, false, true>(),
      make_bvariant<32, 16, 2, false, true>(), make_bvariant<32, 8, 3, false, false, true>(),
      make_bvariant<32, 16, 2, false, false, true>(), make_bvariant<32, 8, 3, false, true, true>(),
      make_bvariant<32, 16, 2, false, 2, true>(), make_bvariant<32, 8, 3, false, 2, true>(),
      make_bvariant<32, 16, 2, false, 2, false>()};
  return v;
}

// Parallel FFT branches of a batch step graph (one stream per branch).
constexpr int kFftBranches = 16;

// The solves are split into lanes whose step chains (FFT branches -> rate
// -> dt -> update) are separate branches of the step graph, the second
// lane one FFT phase behind the first: one lane's cuFFT chains (small
// grids, mostly latency) then run while the other lane's rate kernel fills
// the SMs.  Each shape group's solves stay in one lane (one batched plan).
constexpr int kLanes = 2;

struct Lane {
  int s0 = 0, ns = 0;             // positions [s0, s0 + ns) of the lane order
  int tile0 = 0, ntiles = 0;      // the lane's tiles (current variant)
  int chunk0 = 0, nchunks = 0;    // the lane's update chunks
  std::vector<int> order;         // the lane's shape groups, largest first
  int aux0 = 0, naux = 0;         // its FFT branch streams aux[aux0, aux0 + naux)
  cudaEvent_t fork = nullptr;
};

struct ShapeGroup {
  int ny, nx, count;
  int64_t s_off, k_off, nk;
  cufftHandle fwd = 0, inv = 0;
  float *bk = nullptr;
};

}  // namespace pf5d

using namespace pf5d;

struct pf5d_batch {
  std::vector<BSolve> solves;
  std::vector<int64_t> pt_off;      // point offset of each solve in hi/lo/dX
  BSolve *d_solves = nullptr;
  float4 *hi = nullptr, *lo = nullptr, *dX = nullptr;
  float *s = nullptr;
  cufftComplex *k = nullptr;
  double *spart = nullptr;
  StepState32 *st = nullptr;
  std::vector<ShapeGroup> groups;
  int total_tiles = 0, total_chunks = 0;
  int variant = 0, upd_grid = 1;
  int lane_grid = 1;                // persistent rate blocks of one lane
  cudaStream_t cap = nullptr;
  double *tile_max = nullptr;       // per-tile max |dX/dt| of the last rate launch
  // Shape groups' FFT chains run as parallel branches of the step graph:
  // forked from the lane's stream onto its `aux` streams (high priority, so
  // their blocks get SM slots as the other lane's rate blocks retire),
  // joined back before the lane's rate kernel.
  std::vector<cudaStream_t> aux;
  std::vector<cudaEvent_t> join;
  // Step kernels read the descriptors in lane order (tiles and chunks are
  // numbered in that order); d_solves keeps the caller's order.
  BSolve *d_lane = nullptr;
  std::vector<int> lane_order;      // caller's index at each lane-order position
  std::vector<Lane> lanes;
  cudaStream_t lane_stream = nullptr;
  cudaEvent_t lane_ev[2] = {nullptr, nullptr};
  std::map<int64_t, cudaGraphExec_t> graphs;
  int64_t total_points = 0;
};

namespace {

// Tiles of all solves under `variant` (configure_batch's tiling).
int batch_tiles_of(const pf5d_batch *h, int variant) {
  const BatchVariant &v = batch_variants()[variant];
  const int nt = v.tx * v.ty;
  int tiles = 0;
  for (const auto &b : h->solves)
    tiles += b.dim == 2 ? ((b.R.nx + v.tx - 1) / v.tx) * ((b.R.ny + v.ty - 1) / v.ty)
                        : (b.R.nx + nt - 1) / nt;
  return tiles;
}

pf5d_status configure_batch(pf5d_batch *h, int variant) {
  const auto &vars = batch_variants();
  PF5D_REQUIRE(variant >= 0 && variant < (int)vars.size(), PF5D_ERR_ARG, "bad variant %d", variant);
  const BatchVariant &v = vars[variant];
  v.set_attrs();
  PF5D_LAUNCHED();
  // Tile grid of every solve for this variant, numbered in lane order.
  const int nt = v.tx * v.ty;
  int tiles = 0;
  for (auto &ln : h->lanes) {
    ln.tile0 = tiles;
    for (int k = ln.s0; k < ln.s0 + ln.ns; ++k) {
      BSolve &b = h->solves[h->lane_order[k]];
      if (b.dim == 2) {
        b.ntx = (b.R.nx + v.tx - 1) / v.tx;
        b.nty = (b.R.ny + v.ty - 1) / v.ty;
      } else {
        b.ntx = (b.R.nx + nt - 1) / nt;
        b.nty = 1;
      }
      b.tile0 = tiles;
      b.ntiles = b.ntx * b.nty;
      tiles += b.ntiles;
    }
    ln.ntiles = tiles - ln.tile0;
  }
  h->total_tiles = tiles;
  std::vector<BSolve> lane(h->lane_order.size());
  for (size_t k = 0; k < lane.size(); ++k) lane[k] = h->solves[h->lane_order[k]];
  PF5D_CUDA(cudaMemcpy(h->d_solves, h->solves.data(), h->solves.size() * sizeof(BSolve),
                       cudaMemcpyHostToDevice));
  PF5D_CUDA(cudaMemcpy(h->d_lane, lane.data(), lane.size() * sizeof(BSolve),
                       cudaMemcpyHostToDevice));
  // each lane's rate kernel holds at most its share of the resident block
  // slots, so the other lane's FFT kernels find free slots
  const int per_sm = std::max(1, v.occupancy());
  h->lane_grid = std::max(1, sm_count() * per_sm / (int)std::max<size_t>(h->lanes.size(), 1));
  h->variant = variant;
  return PF5D_OK;
}

// One step of lane L on stream s.  `offset` (optional) is recorded on s
// once the lane's FFT branches have joined.
pf5d_status enqueue_lane_step(pf5d_batch *h, int L, cudaStream_t s, cudaEvent_t offset) {
  const Lane &ln = h->lanes[L];
  const int na = std::min<int>((int)ln.order.size(), ln.naux);
  if (na > 0) {
    PF5D_CUDA(cudaEventRecord(ln.fork, s));
    for (int a = 0; a < na; ++a) PF5D_CUDA(cudaStreamWaitEvent(h->aux[ln.aux0 + a], ln.fork, 0));
  }
  for (int j = 0; j < (int)ln.order.size(); ++j) {
    ShapeGroup &g = h->groups[ln.order[j]];
    cudaStream_t gs = h->aux[ln.aux0 + j % na];
    if (cufftSetStream(g.fwd, gs) != CUFFT_SUCCESS ||
        cufftExecR2C(g.fwd, h->s + g.s_off, h->k + g.k_off) != CUFFT_SUCCESS) {
      set_error("batch cuFFT R2C failed");
      return PF5D_ERR_CUFFT;
    }
    const int64_t total = g.nk * g.count;
    kb_bmul<<<grid_for(total, 256), 256, 0, gs>>>(h->k + g.k_off, g.bk, g.nk, total);
    PF5D_LAUNCHED();
    if (cufftSetStream(g.inv, gs) != CUFFT_SUCCESS ||
        cufftExecC2R(g.inv, h->k + g.k_off, h->s + g.s_off) != CUFFT_SUCCESS) {
      set_error("batch cuFFT C2R failed");
      return PF5D_ERR_CUFFT;
    }
  }
  for (int a = 0; a < na; ++a) {
    PF5D_CUDA(cudaEventRecord(h->join[ln.aux0 + a], h->aux[ln.aux0 + a]));
    PF5D_CUDA(cudaStreamWaitEvent(s, h->join[ln.aux0 + a], 0));
  }
  if (offset) PF5D_CUDA(cudaEventRecord(offset, s));
  const BSolve *ls = h->d_lane + ln.s0;
  batch_variants()[h->variant].launch(std::max(1, std::min(ln.ntiles, h->lane_grid)), s, ls, ln.ns,
                                      ln.tile0, ln.tile0 + ln.ntiles, h->tile_max);
  PF5D_LAUNCHED();
  PF5D_CUDA(launch_pdl(kb_dt, dim3((unsigned)((ln.ns + 7) / 8)), dim3(256), 0, s, ls, ln.ns,
                       (const double *)h->tile_max));
  PF5D_CUDA(launch_pdl(kb_update, dim3((unsigned)std::max(1, std::min(ln.nchunks, h->upd_grid))),
                       dim3(kUpdThreads), 0, s, ls, ln.ns, ln.chunk0, ln.chunk0 + ln.nchunks));
  PF5D_LAUNCHED();
  return PF5D_OK;
}

void drop_graphs(pf5d_batch *h) {
  for (auto &kv : h->graphs) cudaGraphExecDestroy(kv.second);
  h->graphs.clear();
}

pf5d_status batch_graph(pf5d_batch *h, int64_t n, cudaGraphExec_t *out) {
  auto it = h->graphs.find(n);
  if (it != h->graphs.end()) {
    *out = it->second;
    return PF5D_OK;
  }
  cudaGraph_t g = nullptr;
  const bool two = h->lanes.size() > 1;
  PF5D_CUDA(cudaStreamBeginCapture(h->cap, cudaStreamCaptureModeThreadLocal));
  pf5d_status st = PF5D_OK;
  cudaError_t e = cudaSuccess;
  if (two) {
    // the second lane joins the capture, then starts after the first lane's
    // first FFT phase
    e = cudaEventRecord(h->lane_ev[0], h->cap);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(h->lane_stream, h->lane_ev[0], 0);
  }
  for (int64_t i = 0; i < n && st == PF5D_OK && e == cudaSuccess; ++i) {
    st = enqueue_lane_step(h, 0, h->cap, two && i == 0 ? h->lane_ev[1] : nullptr);
    if (st == PF5D_OK && two) {
      if (i == 0) e = cudaStreamWaitEvent(h->lane_stream, h->lane_ev[1], 0);
      if (e == cudaSuccess) st = enqueue_lane_step(h, 1, h->lane_stream, nullptr);
    }
  }
  if (two && st == PF5D_OK && e == cudaSuccess) {
    e = cudaEventRecord(h->lane_ev[0], h->lane_stream);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(h->cap, h->lane_ev[0], 0);
  }
  const cudaError_t e_end = cudaStreamEndCapture(h->cap, &g);
  if (e == cudaSuccess) e = e_end;
  if (st != PF5D_OK || e != cudaSuccess) {
    if (g) cudaGraphDestroy(g);
    if (st != PF5D_OK) return st;
    PF5D_REQUIRE(false, PF5D_ERR_CUDA, "graph capture: %s", cudaGetErrorString(e));
  }
  cudaGraphExec_t exec = nullptr;
  e = cudaGraphInstantiateWithFlags(&exec, g, cudaGraphInstantiateFlagUseNodePriority);
  cudaGraphDestroy(g);
  PF5D_REQUIRE(e == cudaSuccess, PF5D_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(e));
  h->graphs[n] = exec;
  *out = exec;
  return PF5D_OK;
}

}  // namespace

extern "C" {

pf5d_status pf5d_batch_destroy(pf5d_batch *h);

pf5d_status pf5d_batch_create(const pf5d_batch_solve *solves, int32_t nsolves,
                              const float *const *tables32, int32_t ntables, int32_t table_n,
                              double resolution, const double *node_coord, void *stream,
                              pf5d_batch **out) {
  PF5D_REQUIRE(solves && nsolves > 0 && tables32 && ntables > 0 && node_coord && out, PF5D_ERR_ARG,
               "bad arguments");
  auto *h = new pf5d_batch();
  auto fail = [&](pf5d_status code) {
    pf5d_batch_destroy(h);
    return code;
  };
  // --- sizes and groups ------------------------------------------------------
  int64_t npts_total = 0, nchunks_total = 0;
  std::map<std::pair<int, int>, std::vector<int>> by_shape;
  for (int i = 0; i < nsolves; ++i) {
    const pf5d_batch_solve &q = solves[i];
    if (q.dim < 1 || q.dim > 2 || q.table < 0 || q.table >= ntables || !(q.X || (q.hi && q.lo))) {
      set_error("solve %d: batched solves must be 1D or 2D with a valid table and field", i);
      return fail(PF5D_ERR_ARG);
    }
    const int64_t np = q.dim == 1 ? q.shape[0] : q.shape[0] * q.shape[1];
    if (np <= 0 || q.shape[0] <= 0 || (q.dim == 2 && q.shape[1] <= 0)) {
      set_error("solve %d: bad shape", i);
      return fail(PF5D_ERR_ARG);
    }
    if (q.elastic && !q.bk) {
      set_error("solve %d: elastic term needs B(k)", i);
      return fail(PF5D_ERR_ARG);
    }
    h->pt_off.push_back(npts_total);
    npts_total += np;
    nchunks_total += (np + kChunk - 1) / kChunk;
    if (q.dim == 2 && q.elastic) by_shape[{(int)q.shape[0], (int)q.shape[1]}].push_back(i);
  }
  h->total_points = npts_total;
  // s layout: 2D elastic solves contiguous per shape group first, then the rest.
  std::vector<int64_t> s_off(nsolves, -1);
  std::vector<std::vector<int>> members;     // solves of each shape group
  int64_t s_total = 0, k_total = 0;
  for (auto &kv : by_shape) {
    ShapeGroup g;
    g.ny = kv.first.first;
    g.nx = kv.first.second;
    g.count = (int)kv.second.size();
    g.s_off = s_total;
    g.nk = (int64_t)g.ny * (g.nx / 2 + 1);
    g.k_off = k_total;
    for (int idx : kv.second) {
      s_off[idx] = s_total;
      s_total += (int64_t)g.ny * g.nx;
    }
    k_total += g.nk * g.count;
    h->groups.push_back(g);
    members.push_back(kv.second);
  }
  for (int i = 0; i < nsolves; ++i)
    if (s_off[i] < 0) {
      s_off[i] = s_total;
      s_total += solves[i].dim == 1 ? solves[i].shape[0] : solves[i].shape[0] * solves[i].shape[1];
    }
  if (cudaMalloc(&h->hi, npts_total * sizeof(float4)) != cudaSuccess ||
      cudaMalloc(&h->lo, npts_total * sizeof(float4)) != cudaSuccess ||
      cudaMalloc(&h->dX, npts_total * sizeof(float4)) != cudaSuccess ||
      cudaMalloc(&h->s, std::max<int64_t>(s_total, 1) * sizeof(float)) != cudaSuccess ||
      cudaMalloc(&h->k, std::max<int64_t>(k_total, 1) * sizeof(cufftComplex)) != cudaSuccess ||
      cudaMalloc(&h->spart, std::max<int64_t>(nchunks_total, 1) * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&h->st, nsolves * sizeof(StepState32)) != cudaSuccess ||
      cudaMalloc(&h->d_solves, nsolves * sizeof(BSolve)) != cudaSuccess ||
      cudaMalloc(&h->d_lane, nsolves * sizeof(BSolve)) != cudaSuccess ||
      cudaStreamCreateWithFlags(&h->cap, cudaStreamNonBlocking) != cudaSuccess) {
    set_error("device allocation failed");
    return fail(PF5D_ERR_CUDA);
  }
  // --- cuFFT groups ----------------------------------------------------------
  for (auto &g : h->groups) {
    long long n2[2] = {g.ny, g.nx};
    size_t ws = 0;
    const long long idist = (long long)g.ny * g.nx, odist = g.nk;
    if (cufftCreate(&g.fwd) != CUFFT_SUCCESS || cufftCreate(&g.inv) != CUFFT_SUCCESS ||
        cufftMakePlanMany64(g.fwd, 2, n2, nullptr, 1, idist, nullptr, 1, odist, CUFFT_R2C, g.count,
                            &ws) != CUFFT_SUCCESS ||
        cufftMakePlanMany64(g.inv, 2, n2, nullptr, 1, odist, nullptr, 1, idist, CUFFT_C2R, g.count,
                            &ws) != CUFFT_SUCCESS) {
      set_error("cuFFT plan creation failed for %dx%d", g.ny, g.nx);
      return fail(PF5D_ERR_CUFFT);
    }
    // B(k) of the first solve of the group (the same for all: it depends only
    // on the direction of k), scaled by 1/N.
    const pf5d_batch_solve *first = nullptr;
    for (int i = 0; i < nsolves && !first; ++i)
      if (solves[i].dim == 2 && solves[i].elastic && solves[i].shape[0] == g.ny &&
          solves[i].shape[1] == g.nx)
        first = &solves[i];
    std::vector<float> b(g.nk);
    const double inv_n = 1.0 / (double)((int64_t)g.ny * g.nx);
    for (int64_t i = 0; i < g.nk; ++i) b[i] = (float)(first->bk[i] * inv_n);
    if (cudaMalloc(&g.bk, g.nk * sizeof(float)) != cudaSuccess ||
        cudaMemcpy(g.bk, b.data(), g.nk * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess) {
      set_error("device allocation failed");
      return fail(PF5D_ERR_CUDA);
    }
  }
  // --- lanes: shape groups largest first to the lighter lane, then the
  //     solves without an FFT; FFT branch streams split between the lanes --
  std::vector<int> gorder;
  for (int j = 0; j < (int)h->groups.size(); ++j) gorder.push_back(j);
  std::stable_sort(gorder.begin(), gorder.end(), [&](int a, int b) {
    const auto &ga = h->groups[a], &gb = h->groups[b];
    return (int64_t)ga.ny * ga.nx * ga.count > (int64_t)gb.ny * gb.nx * gb.count;
  });
  const int nl = nsolves >= 2 ? kLanes : 1;
  std::vector<int> lane_of(nsolves, -1);
  std::vector<int64_t> lane_pts(nl, 0);
  std::vector<std::vector<int>> lane_groups(nl);
  auto lighter = [&]() {
    return (int)(std::min_element(lane_pts.begin(), lane_pts.end()) - lane_pts.begin());
  };
  for (int j : gorder) {
    const int L = lighter();
    lane_groups[L].push_back(j);
    lane_pts[L] += (int64_t)h->groups[j].ny * h->groups[j].nx * h->groups[j].count;
    for (int i : members[j]) lane_of[i] = L;
  }
  for (int i = 0; i < nsolves; ++i)
    if (lane_of[i] < 0) {
      const int L = lighter();
      lane_of[i] = L;
      lane_pts[L] += solves[i].dim == 1 ? solves[i].shape[0] : solves[i].shape[0] * solves[i].shape[1];
    }
  int least_pri = 0, greatest_pri = 0;
  if (cudaDeviceGetStreamPriorityRange(&least_pri, &greatest_pri) != cudaSuccess) {
    set_error("stream priority query failed");
    return fail(PF5D_ERR_CUDA);
  }
  const int per_lane = std::max(1, kFftBranches / nl);
  for (int L = 0; L < nl; ++L) {
    Lane ln;
    ln.s0 = (int)h->lane_order.size();
    for (int i = 0; i < nsolves; ++i)
      if (lane_of[i] == L) h->lane_order.push_back(i);
    ln.ns = (int)h->lane_order.size() - ln.s0;
    if (ln.ns == 0) continue;
    ln.order = lane_groups[L];
    ln.aux0 = (int)h->aux.size();
    ln.naux = std::min<int>((int)ln.order.size(), per_lane);
    h->lanes.push_back(ln);             // registered first: teardown frees what follows
    if (ln.naux > 0 &&
        cudaEventCreateWithFlags(&h->lanes.back().fork, cudaEventDisableTiming) != cudaSuccess) {
      set_error("event creation failed");
      return fail(PF5D_ERR_CUDA);
    }
    for (int a = 0; a < ln.naux; ++a) {
      cudaStream_t as = nullptr;
      cudaEvent_t ev = nullptr;
      if (cudaStreamCreateWithPriority(&as, cudaStreamNonBlocking, greatest_pri) != cudaSuccess) {
        set_error("stream creation failed");
        return fail(PF5D_ERR_CUDA);
      }
      h->aux.push_back(as);
      if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess) {
        set_error("event creation failed");
        return fail(PF5D_ERR_CUDA);
      }
      h->join.push_back(ev);
    }
  }
  if (h->lanes.size() > 1 &&
      (cudaStreamCreateWithFlags(&h->lane_stream, cudaStreamNonBlocking) != cudaSuccess ||
       cudaEventCreateWithFlags(&h->lane_ev[0], cudaEventDisableTiming) != cudaSuccess ||
       cudaEventCreateWithFlags(&h->lane_ev[1], cudaEventDisableTiming) != cudaSuccess)) {
    set_error("stream creation failed");
    return fail(PF5D_ERR_CUDA);
  }
  // --- per-solve descriptors -------------------------------------------------
  int64_t chunk = 0;
  std::vector<StepState32> init(nsolves);
  for (int i = 0; i < nsolves; ++i) {
    const pf5d_batch_solve &q = solves[i];
    BSolve b{};
    Rate32 &P = b.R;
    b.dim = q.dim;
    if (q.dim == 1) {
      P.nz = 1; P.ny = 1; P.nx = (int)q.shape[0];
    } else {
      P.nz = 1; P.ny = (int)q.shape[0]; P.nx = (int)q.shape[1];
    }
    b.npts = q.dim == 1 ? q.shape[0] : q.shape[0] * q.shape[1];
    b.hi = h->hi + h->pt_off[i];
    b.lo = h->lo + h->pt_off[i];
    b.s = h->s + s_off[i];
    b.spart = h->spart + chunk;
    b.nchunks = (int)((b.npts + kChunk - 1) / kChunk);
    chunk += b.nchunks;
    b.emode = !q.elastic ? 0 : (q.dim == 1 ? 1 : 2);
    b.bn = (q.elastic && q.dim == 1) ? (float)q.bk[1 % (q.shape[0] / 2 + 1)] : 0.f;
    b.oob_interval = q.oob_interval;
    P.D = b.hi;
    P.sp = q.elastic ? b.s : nullptr;
    P.dX = h->dX + h->pt_off[i];
    Table32 &T = P.T;
    T.grid = tables32[q.table];
    T.coord = node_coord;
    T.n = table_n;
    T.stride = kStride32;
    T.inv_step = 1.0 / resolution;
    T.inv_step_f = (float)T.inv_step;
    T.threshold = 1.0 - 4.0 * resolution - 1e-9;
    T.max_nn_dist = q.max_nn_dist;
    double sx = 0.0;
    for (int c = 0; c < S; ++c) {
      const double u = q.x0[c] * T.inv_step;
      const double fl = floor(u);
      T.ib[c] = (int)fl;
      T.fb[c] = (float)(u - fl);
      T.x0[c] = q.x0[c];
      sx = sx + q.x0[c];
      P.kappa[c] = (float)q.kappa[c];
      P.lvec[c] = (float)q.lvec[c];
      P.x0f[c] = (float)q.x0[c];
      b.lvec[c] = (float)q.lvec[c];
      b.x0[c] = q.x0[c];
    }
    T.sum_x0 = sx;
    b.sum_x0 = sx;
    P.c_fe = 1.0 - sx;
    P.flux_scale = (float)(0.5 / (q.dx * q.dx));
    P.inv_dx2 = (float)(1.0 / (q.dx * q.dx));
    P.ctld = q.ctld;
    P.t_cfl = q.t_cfl;
    P.lower = q.lower_limit;
    P.upper = q.upper_limit;
    P.factor = q.max_change_factor;
    P.adaptive = q.adaptive;
    P.st = h->st + i;
    init[i] = StepState32{};
    init[i].dt = q.dt0;
    if (q.hi && q.lo) {
      init[i].time = q.time0;
      init[i].step = q.step0;
    }
    h->solves.push_back(b);
  }
  h->total_chunks = (int)chunk;
  // update chunks numbered in lane order (b.spart keeps the solve's own
  // partial-sum region)
  int run = 0;
  for (auto &ln : h->lanes) {
    ln.chunk0 = run;
    for (int k = ln.s0; k < ln.s0 + ln.ns; ++k) {
      BSolve &b = h->solves[h->lane_order[k]];
      b.chunk0 = run;
      run += b.nchunks;
    }
    ln.nchunks = run - ln.chunk0;
  }
  h->upd_grid = std::min<int>(h->total_chunks, sm_count() * 8);
  cudaStream_t s = as_stream(stream);
  if (cudaMemcpy(h->st, init.data(), nsolves * sizeof(StepState32), cudaMemcpyHostToDevice) !=
      cudaSuccess) {
    set_error("state upload failed");
    return fail(PF5D_ERR_CUDA);
  }
  int max_tiles = 1;
  for (int v = 0; v < (int)batch_variants().size(); ++v)
    max_tiles = std::max(max_tiles, batch_tiles_of(h, v));
  if (cudaMalloc(&h->tile_max, (size_t)max_tiles * sizeof(double)) != cudaSuccess) {
    set_error("device allocation failed");
    return fail(PF5D_ERR_CUDA);
  }
  pf5d_status st = configure_batch(h, 0);
  if (st != PF5D_OK) return fail(st);
  for (int i = 0; i < nsolves; ++i) {
    const unsigned g = std::max(1, std::min(h->solves[i].nchunks, 1024));
    if (solves[i].hi && solves[i].lo)
      kb_resume<<<g, kUpdThreads, 0, s>>>(reinterpret_cast<const float4 *>(solves[i].hi),
                                          reinterpret_cast<const float4 *>(solves[i].lo),
                                          h->d_solves, i);
    else
      kb_split<<<g, kUpdThreads, 0, s>>>(solves[i].X, h->d_solves, i);
    if (cudaGetLastError() != cudaSuccess) {
      set_error("split launch failed");
      return fail(PF5D_ERR_CUDA);
    }
  }
  if (cudaStreamSynchronize(s) != cudaSuccess) {
    set_error("initial state failed");
    return fail(PF5D_ERR_CUDA);
  }
  *out = h;
  return PF5D_OK;
}

pf5d_status pf5d_batch_advance(pf5d_batch *h, int64_t nsteps, void *stream) {
  PF5D_REQUIRE(h && nsteps >= 0, PF5D_ERR_ARG, "bad arguments");
  cudaStream_t s = as_stream(stream);
  while (nsteps > 0) {
    const int64_t n = nsteps < 25 ? nsteps : 25;
    cudaGraphExec_t g = nullptr;
    pf5d_status st = batch_graph(h, n, &g);
    if (st != PF5D_OK) return st;
    PF5D_CUDA(cudaGraphLaunch(g, s));
    nsteps -= n;
  }
  return PF5D_OK;
}

pf5d_status pf5d_batch_states(pf5d_batch *h, pf5d_step_state *out, void *stream) {
  PF5D_REQUIRE(h && out, PF5D_ERR_ARG, "bad arguments");
  std::vector<StepState32> hs(h->solves.size());
  cudaStream_t s = as_stream(stream);
  PF5D_CUDA(cudaMemcpyAsync(hs.data(), h->st, hs.size() * sizeof(StepState32),
                            cudaMemcpyDeviceToHost, s));
  PF5D_CUDA(cudaStreamSynchronize(s));
  for (size_t i = 0; i < hs.size(); ++i) {
    out[i].dt = hs[i].dt;
    out[i].time = hs[i].time;
    out[i].xdotmax = hs[i].xdotmax;
    out[i].step = hs[i].step;
    out[i].flags = hs[i].flags | (hs[i].halt ? PF5D_FLAG_HALTED : 0u);
    out[i].halted = hs[i].halt;
  }
  return PF5D_OK;
}

pf5d_status pf5d_batch_field(pf5d_batch *h, int32_t i, double *X_out, void *stream) {
  PF5D_REQUIRE(h && X_out && i >= 0 && i < (int)h->solves.size(), PF5D_ERR_ARG, "bad arguments");
  kb_join<<<grid_for(h->solves[i].npts, 256, 2), 256, 0, as_stream(stream)>>>(h->d_solves, i,
                                                                              X_out);
  PF5D_LAUNCHED();
  return PF5D_OK;
}

pf5d_status pf5d_batch_export(pf5d_batch *h, int32_t i, float *hi_out, float *lo_out,
                              void *stream) {
  PF5D_REQUIRE(h && hi_out && lo_out && i >= 0 && i < (int)h->solves.size(), PF5D_ERR_ARG,
               "bad arguments");
  const BSolve &b = h->solves[i];
  cudaStream_t s = as_stream(stream);
  PF5D_CUDA(cudaMemcpyAsync(hi_out, b.hi, b.npts * sizeof(float4), cudaMemcpyDeviceToDevice, s));
  PF5D_CUDA(cudaMemcpyAsync(lo_out, b.lo, b.npts * sizeof(float4), cudaMemcpyDeviceToDevice, s));
  return PF5D_OK;
}

pf5d_status pf5d_batch_set_variant(pf5d_batch *h, int32_t variant) {
  PF5D_REQUIRE(h, PF5D_ERR_ARG, "null batch");
  pf5d_status st = configure_batch(h, variant);
  if (st == PF5D_OK) drop_graphs(h);
  return st;
}

int32_t pf5d_batch_variant_count(void) { return (int32_t)batch_variants().size(); }

pf5d_status pf5d_batch_autotune(pf5d_batch *h, int32_t *variant, float *best_ms, void *stream) {
  PF5D_REQUIRE(h, PF5D_ERR_ARG, "null batch");
  cudaStream_t s = as_stream(stream);
  const size_t n = h->solves.size();
  std::vector<StepState32> saved(n);
  PF5D_CUDA(cudaMemcpyAsync(saved.data(), h->st, n * sizeof(StepState32), cudaMemcpyDeviceToHost, s));
  PF5D_CUDA(cudaStreamSynchronize(s));
  cudaEvent_t e0, e1;
  PF5D_CUDA(cudaEventCreate(&e0));
  PF5D_CUDA(cudaEventCreate(&e1));
  int best = h->variant;
  float best_t = 1e30f;
  for (int v = 0; v < (int)batch_variants().size(); ++v) {
    if (configure_batch(h, v) != PF5D_OK) continue;
    const int grid = std::max(h->total_tiles, 1);
    batch_variants()[v].launch(grid, s, h->d_lane, (int)n, 0, h->total_tiles, h->tile_max);
    if (cudaGetLastError() != cudaSuccess) continue;
    PF5D_CUDA(cudaEventRecord(e0, s));
    for (int r = 0; r < 3; ++r)
      batch_variants()[v].launch(grid, s, h->d_lane, (int)n, 0, h->total_tiles, h->tile_max);
    PF5D_CUDA(cudaEventRecord(e1, s));
    PF5D_CUDA(cudaEventSynchronize(e1));
    float ms = 0.f;
    PF5D_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    if (ms / 3 < best_t) {
      best_t = ms / 3;
      best = v;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  pf5d_status st = configure_batch(h, best);
  if (st != PF5D_OK) return st;
  drop_graphs(h);
  PF5D_CUDA(cudaMemcpyAsync(h->st, saved.data(), n * sizeof(StepState32), cudaMemcpyHostToDevice, s));
  PF5D_CUDA(cudaStreamSynchronize(s));
  if (variant) *variant = best;
  if (best_ms) *best_ms = best_t;
  return PF5D_OK;
}

pf5d_status pf5d_batch_destroy(pf5d_batch *h) {
  if (!h) return PF5D_OK;
  drop_graphs(h);
  for (auto &g : h->groups) {
    if (g.fwd) cufftDestroy(g.fwd);
    if (g.inv) cufftDestroy(g.inv);
    cudaFree(g.bk);
  }
  cudaFree(h->hi);
  cudaFree(h->lo);
  cudaFree(h->dX);
  cudaFree(h->s);
  cudaFree(h->k);
  cudaFree(h->spart);
  cudaFree(h->st);
  cudaFree(h->d_solves);
  cudaFree(h->d_lane);
  cudaFree(h->tile_max);
  if (h->cap) cudaStreamDestroy(h->cap);
  for (auto as : h->aux) cudaStreamDestroy(as);
  for (auto ev : h->join) cudaEventDestroy(ev);
  for (auto &ln : h->lanes)
    if (ln.fork) cudaEventDestroy(ln.fork);
  if (h->lane_stream) cudaStreamDestroy(h->lane_stream);
  for (auto ev : h->lane_ev)
    if (ev) cudaEventDestroy(ev);
  delete h;
  return PF5D_OK;
}

}  // extern "C"
