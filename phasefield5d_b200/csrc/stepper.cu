// stepper.cu -- the FP64 step loop of examples/simulate.py:230-320 (saves
// off) as a device-resident stepper.
//
// Per step (all on one stream, replayed from a CUDA graph):
//   1. cuFFT D2Z of the misfit scalar s      (s written by step 4 of the
//      previous step, or by k_misfit at start)
//   2. k_bmul: S(k) *= B(k)/N
//   3. cuFFT Z2D -> s'(x)
//   4. k_rate_*: fused chemical potential + flux divergence.  Per tile of a
//      plane (x fastest), marching plane by plane along axis 0:
//        - X planes with a 2-cell halo staged in shared memory (ring of 3),
//        - mu and M at the tile plus a 1-cell halo (ring of 2 planes):
//          table interpolation (nearest-row fallback), periodic Laplacian,
//          mu = (mu_chem - lap*kappa) + s'*l,
//        - one flux per face (the +axis0 face of the previous plane is kept
//          in registers and reused as this plane's -axis0 face),
//        - dX/dt written once; each block stores its max |dX/dt| in its
//          own slot (plain store).
//      Variants (autotuned, all computing the same values): tile shapes,
//      a split form (k_chem64 writes mu/M once per point, the tile kernel
//      reads them back), table-cell sort, shared table window, per-point
//      faces.
//   5. k_dt_finish (one block): max over the slots, the adaptive dt rule,
//      dt / time / step advanced on the device.
//   6. k_update_step: X += dX*dt; clamp; s for the next step; every
//      oob_interval steps the out_of_bounds test, which halts the stepper
//      (every later kernel returns at entry) on a hard violation.
//
// Every FP64 operation follows the reference's order; the unit is compiled
// with -fmad=false, so apart from the FFT (cuFFT vs pocketfft rounding) the
// trajectory equals the reference's bit for bit.
#include <algorithm>
#include <cstring>
#include <map>
#include <vector>

#include <cuda_pipeline_primitives.h>

#include "pf5d_device.cuh"
#include "pf5d_fft.h"
#include "pf5d_fp32c.h"
#include "pf5d_tiles.cuh"
#include "pf5d_window.cuh"
#include "pf5d_diag.cuh"

namespace pf5d {

struct StepState {
  double dt;
  double time;
  double xdotmax;      // max |dX/dt| of the last rate evaluation
  unsigned flags;      // PF5D_FLAG_* accumulated
  unsigned halt;       // non-zero: every step kernel returns at entry
  long long step;      // completed steps
};

struct RateParams {
  int nz, ny, nx;              // 3D: (n0, n1, n2); 2D: (1, n0, n1); 1D: (1, 1, n0)
  const double *X;
  const double *sp;            // s' (already scaled by 1/N) or nullptr
  double *dX;
  Table T;
  Vec4 kappa, lvec;
  double inv_dx, inv_dx2;
  double ctld, t_cfl, lower, upper, factor;
  int adaptive;
  StepState *st;
  double *mm;                  // split rate: mu_1..4, M_Fe, M_1..4 per point, SoA [NP][npts]
  int64_t npts;
  double *partial;             // per-block max |dX/dt| of the last rate launch
};

// ------------------------------------------------------------------------
// Shared pieces of the rate kernels
// ------------------------------------------------------------------------

// chemical potential and mobility at one point (examples/simulate.py:242-258).
template <bool VEC>
__device__ __forceinline__ void chem_point(const RateParams &P, const double x[S],
                                           const double lap[S], double spv, double mu[S],
                                           double M[NM], unsigned *flags) {
  double v[NP];
  interp_point<VEC>(P.T, x, v, flags);
#pragma unroll
  for (int c = 0; c < S; ++c) {
    const double lk = lap[c] * P.kappa.v[c];
    double m = v[c] - lk;
    if (P.sp) m = m + spv * P.lvec.v[c];
    mu[c] = m;
  }
#pragma unroll
  for (int c = 0; c < NM; ++c) M[c] = v[S + c];
}

constexpr int kWin64 = 3;                       // window nodes per axis (2 cells)
constexpr int kWinNodes64 = kWin64 * kWin64 * kWin64 * kWin64;
constexpr int kNodeV64 = 5;                     // double2 per 10-double table node

// Table cell of x exactly as the reference computes it (interpolation.py:103-121).
__device__ __forceinline__ bool cell64(const Table &T, const double x[S], int ii[S], double tt[S]) {
  if (!linear_region(T, x)) return false;
#pragma unroll
  for (int a = 0; a < S; ++a) axis_coord(x[a] * T.inv_step, T.n, ii[a], tt[a]);
  return true;
}

// The 16-corner sum of interp_linear<true> from node-strided double2 data
// (global table or shared window); identical arithmetic and order.
__device__ __forceinline__ void interp_nodes64(const double2 *base, int64_t s0, int64_t s1,
                                               int64_t s2, int64_t s3, const double tt[S],
                                               double out[NP]) {
  const double q0 = 1.0 - tt[0], q1 = 1.0 - tt[1], q2 = 1.0 - tt[2], q3 = 1.0 - tt[3];
#pragma unroll
  for (int c = 0; c < 16; ++c) {
    const int b0 = (c >> 3) & 1, b1 = (c >> 2) & 1, b2 = (c >> 1) & 1, b3 = c & 1;
    const double w = (b0 ? tt[0] : q0) * (b1 ? tt[1] : q1) * (b2 ? tt[2] : q2) * (b3 ? tt[3] : q3);
    const double2 *node = base + b0 * s0 + b1 * s1 + b2 * s2 + b3 * s3;
    double v[NP + 1];
#pragma unroll
    for (int k = 0; k < kNodeV64; ++k) {
      const double2 a = node[k];
      v[2 * k] = a.x;
      v[2 * k + 1] = a.y;
    }
#pragma unroll
    for (int p = 0; p < NP; ++p) {
      const double term = w * v[p];
      out[p] = (c == 0) ? term : out[p] + term;
    }
  }
}

// Table value at x with the shared window (VEC tables only): window when the
// cell fits, global table otherwise, nearest row outside the linear region.
template <bool VEC>
__device__ __forceinline__ void interp_win64(const Table &T, const double x[S], const double2 *win,
                                             const int *win_lo, double out[NP], unsigned *flags) {
  if (!VEC) {
    interp_point<false>(T, x, out, flags);
    return;
  }
  int ii[S];
  double tt[S];
  if (cell64(T, x, ii, tt)) {
    const int off = win ? window_cell<kWin64>(ii, win_lo) : -1;
    if (off >= 0) {
      constexpr int w3 = kNodeV64, w2 = kWin64 * w3, w1 = kWin64 * w2, w0 = kWin64 * w1;
      interp_nodes64(win + off * kNodeV64, w0, w1, w2, w3, tt, out);
    } else {
      const int64_t s3 = kNodeV64, s2 = (int64_t)T.n * s3, s1 = (int64_t)T.n * s2,
                    s0 = (int64_t)T.n * s1;
      const double2 *g = reinterpret_cast<const double2 *>(T.grid);
      interp_nodes64(g + ii[0] * s0 + ii[1] * s1 + ii[2] * s2 + ii[3] * s3, s0, s1, s2, s3, tt,
                     out);
    }
    return;
  }
  const NearestNode r = nearest_node(T, x[0], x[1], x[2], x[3]);
  *flags |= r.flags;
  const double *row = T.grid + (r.node < 0 ? 0 : r.node) * T.stride;
#pragma unroll
  for (int p = 0; p < NP; ++p)
    out[p] = r.node < 0 ? __longlong_as_double(0x7ff8000000000000LL) : __ldg(row + p);
}

// Table values at two points at once (VEC tables): when both lie in the
// linear region of one table cell, each corner node is loaded once and its
// terms accumulated into both -- the same weights and left-to-right sums as
// interp_nodes64, so the same bits; otherwise each point takes interp_win64's
// path without a window.  hasB = false evaluates A alone.
__device__ __forceinline__ void interp_pair64(const Table &T, const double xA[S],
                                              const double xB[S], bool hasB, double vA[NP],
                                              double vB[NP], unsigned *flags) {
  int iA[S], iB[S];
  double tA[S], tB[S];
  const bool linA = cell64(T, xA, iA, tA);
  const bool linB = hasB && cell64(T, xB, iB, tB);
  if (linA && linB && iA[0] == iB[0] && iA[1] == iB[1] && iA[2] == iB[2] && iA[3] == iB[3]) {
    const int64_t s3 = kNodeV64, s2 = (int64_t)T.n * s3, s1 = (int64_t)T.n * s2,
                  s0 = (int64_t)T.n * s1;
    const double2 *base = reinterpret_cast<const double2 *>(T.grid) + iA[0] * s0 + iA[1] * s1 +
                          iA[2] * s2 + iA[3] * s3;
    const double qA0 = 1.0 - tA[0], qA1 = 1.0 - tA[1], qA2 = 1.0 - tA[2], qA3 = 1.0 - tA[3];
    const double qB0 = 1.0 - tB[0], qB1 = 1.0 - tB[1], qB2 = 1.0 - tB[2], qB3 = 1.0 - tB[3];
#pragma unroll
    for (int c = 0; c < 16; ++c) {
      const int b0 = (c >> 3) & 1, b1 = (c >> 2) & 1, b2 = (c >> 1) & 1, b3 = c & 1;
      const double wA = (b0 ? tA[0] : qA0) * (b1 ? tA[1] : qA1) * (b2 ? tA[2] : qA2) *
                        (b3 ? tA[3] : qA3);
      const double wB = (b0 ? tB[0] : qB0) * (b1 ? tB[1] : qB1) * (b2 ? tB[2] : qB2) *
                        (b3 ? tB[3] : qB3);
      const double2 *node = base + b0 * s0 + b1 * s1 + b2 * s2 + b3 * s3;
      double v[NP + 1];
#pragma unroll
      for (int k = 0; k < kNodeV64; ++k) {
        const double2 a = __ldg(node + k);
        v[2 * k] = a.x;
        v[2 * k + 1] = a.y;
      }
#pragma unroll
      for (int p = 0; p < NP; ++p) {
        const double ta = wA * v[p], tb = wB * v[p];
        vA[p] = (c == 0) ? ta : vA[p] + ta;
        vB[p] = (c == 0) ? tb : vB[p] + tb;
      }
    }
    return;
  }
  const int o[S] = {0, 0, 0, 0};
  interp_win64<true>(T, xA, nullptr, o, vA, flags);
  if (hasB) interp_win64<true>(T, xB, nullptr, o, vB, flags);
}

// Shared-memory scratch of a per-tile cell sort: hist[256], wsum[NT/32+1],
// order/rank/key per mu/M position.
struct SortScratch {
  int *hist;
  int *wsum;
  unsigned short *order;
  unsigned short *rank;
  unsigned char *key;
};

constexpr unsigned short kNoRank = 0xFFFFu;

// mu/M of one plane (tile + 1-cell halo, or tile only) into dst, making the
// table window in `win` current first (win_lo: origin + valid flag).  Xm/Xp: axis-0 neighbour planes (3D) or
// nullptr (2D).  Laplacian neighbour order as operators.py:49-76.  SORT:
// the positions are first put in table-cell order (cell_hash counting
// sort) so the lanes of a warp gather the same table nodes; which thread
// evaluates a position changes, the values do not.
template <int TX, int TY, int DIM, bool VEC, bool WIN, int NTH = TX * TY, int SORT = 0>
__device__ __forceinline__ void mu_plane64(const RateParams &P, const double *Xm, const double *Xc,
                                           const double *Xp, double *dst, int64_t zoff,
                                           const int *wx, const int *wy, bool interior_only,
                                           double2 *win, int *win_lo, unsigned *flags, int tid,
                                           SortScratch ss = {}) {
  using G = PlaneGeom<TX, TY, NTH>;
  auto skip = [&](int mx, int my) {
    const bool ex = (mx == 0 || mx == G::MX - 1), ey = (my == 0 || my == G::MY - 1);
    return interior_only ? (ex || ey) : (ex && ey);
  };
  // Table window around the tile centre's cell (reloaded if it moved).
  bool use_win = false;
  int o[S] = {0, 0, 0, 0};
  if (VEC && WIN) {
    int rep[S];
    double tr[S], xc[S];
    const int cp = (TY / 2 + 2) * G::HX + (TX / 2 + 2);
#pragma unroll
    for (int c = 0; c < S; ++c) xc[c] = Xc[c * G::PX + cp];
    use_win = cell64(P.T, xc, rep, tr);
    if (use_win) {
      window_origin<kWin64>(rep, tr, o);
      ensure_window<kWin64, kNodeV64, double2, G::NT>(reinterpret_cast<const double2 *>(P.T.grid),
                                                       P.T.n, o, win, win_lo, tid);
    }
  }
  int nwork = G::PM;
  if constexpr (SORT) {
    for (int i = tid; i < 256; i += NTH) ss.hist[i] = 0;
    __syncthreads();
    for (int pos = tid; pos < G::PM; pos += NTH) {
      const int my = pos / G::MX, mx = pos - my * G::MX;
      if (skip(mx, my)) {
        ss.rank[pos] = kNoRank;
        continue;
      }
      const int px = (my + 1) * G::HX + (mx + 1);
      double xk[S];
#pragma unroll
      for (int c = 0; c < S; ++c) xk[c] = Xc[c * G::PX + px];
      const int k = cell_hash(xk, (float)P.T.inv_step);
      ss.key[pos] = (unsigned char)k;
      ss.rank[pos] = (unsigned short)atomicAdd(&ss.hist[k], 1);
    }
    __syncthreads();
    nwork = block_exclusive_scan<256, NTH>(ss.hist, ss.wsum, tid);
    for (int pos = tid; pos < G::PM; pos += NTH)
      if (ss.rank[pos] != kNoRank) ss.order[ss.hist[ss.key[pos]] + ss.rank[pos]] = (unsigned short)pos;
    __syncthreads();
  }
  if constexpr (SORT == 2 && VEC) {
    // two consecutive positions of the cell order per thread, corner loads
    // shared when they lie in one table cell (interp_pair64)
    auto inputs = [&](int pos, double x[S], double lap[S], double &spv) {
      const int my = pos / G::MX, mx = pos - my * G::MX;
      const int px = (my + 1) * G::HX + (mx + 1);
#pragma unroll
      for (int c = 0; c < S; ++c) {
        const double *q = Xc + c * G::PX;
        x[c] = q[px];
        if (DIM == 3)
          lap[c] = (Xp[c * G::PX + px] + Xm[c * G::PX + px] + q[px + G::HX] + q[px - G::HX] +
                    q[px + 1] + q[px - 1] - 6.0 * x[c]) * P.inv_dx2;
        else
          lap[c] = (q[px + G::HX] + q[px - G::HX] + q[px + 1] + q[px - 1] - 4.0 * x[c]) * P.inv_dx2;
      }
      spv = P.sp ? __ldg(P.sp + zoff + (int64_t)wy[my + 1] * P.nx + wx[mx + 1]) : 0.0;
    };
    auto store = [&](int pos, const double v[NP], const double lap[S], double spv) {
#pragma unroll
      for (int c = 0; c < S; ++c) {
        const double lk = lap[c] * P.kappa.v[c];
        double m = v[c] - lk;
        if (P.sp) m = m + spv * P.lvec.v[c];
        dst[c * G::PM + pos] = m;
      }
#pragma unroll
      for (int c = 0; c < NM; ++c) dst[(S + c) * G::PM + pos] = v[S + c];
    };
    for (int w = 2 * tid; w < nwork; w += 2 * NTH) {
      const int posA = ss.order[w];
      const bool hasB = w + 1 < nwork;
      const int posB = hasB ? (int)ss.order[w + 1] : posA;
      double xA[S], lapA[S], xB[S], lapB[S], spA, spB, vA[NP], vB[NP];
      inputs(posA, xA, lapA, spA);
      inputs(posB, xB, lapB, spB);
      interp_pair64(P.T, xA, xB, hasB, vA, vB, flags);
      store(posA, vA, lapA, spA);
      if (hasB) store(posB, vB, lapB, spB);
    }
  } else {
  for (int w = tid; w < nwork; w += NTH) {
    const int pos = SORT ? (int)ss.order[w] : w;
    const int my = pos / G::MX, mx = pos - my * G::MX;
    if (!SORT && skip(mx, my)) continue;
    const int px = (my + 1) * G::HX + (mx + 1);
    double x[S], lap[S];
#pragma unroll
    for (int c = 0; c < S; ++c) {
      const double *q = Xc + c * G::PX;
      x[c] = q[px];
      if (DIM == 3)
        lap[c] = (Xp[c * G::PX + px] + Xm[c * G::PX + px] + q[px + G::HX] + q[px - G::HX] +
                  q[px + 1] + q[px - 1] - 6.0 * x[c]) * P.inv_dx2;
      else
        lap[c] = (q[px + G::HX] + q[px - G::HX] + q[px + 1] + q[px - 1] - 4.0 * x[c]) * P.inv_dx2;
    }
    const double spv = P.sp ? __ldg(P.sp + zoff + (int64_t)wy[my + 1] * P.nx + wx[mx + 1]) : 0.0;
    double v[NP];
    interp_win64<VEC>(P.T, x, use_win ? win : nullptr, o, v, flags);
#pragma unroll
    for (int c = 0; c < S; ++c) {
      const double lk = lap[c] * P.kappa.v[c];
      double m = v[c] - lk;
      if (P.sp) m = m + spv * P.lvec.v[c];
      dst[c * G::PM + pos] = m;
    }
#pragma unroll
    for (int c = 0; c < NM; ++c) dst[(S + c) * G::PM + pos] = v[S + c];
  }
  }
}

// mu/M of one plane (tile + 1-cell halo, or tile only) read from the split
// buffer P.mm (written by k_chem64) into dst, in mu_plane64's layout.
template <int TX, int TY, int NTH = TX * TY>
__device__ __forceinline__ void load_mu_plane(const RateParams &P, int64_t zoff, const int *wx,
                                              const int *wy, bool interior_only, double *dst,
                                              int tid) {
  using G = PlaneGeom<TX, TY, NTH>;
  for (int pos = tid; pos < G::PM; pos += G::NT) {
    const int my = pos / G::MX, mx = pos - my * G::MX;
    const bool ex = (mx == 0 || mx == G::MX - 1), ey = (my == 0 || my == G::MY - 1);
    if (interior_only ? (ex || ey) : (ex && ey)) continue;
    const double *src = P.mm + zoff + (int64_t)wy[my + 1] * P.nx + wx[mx + 1];
#pragma unroll
    for (int c = 0; c < NP; ++c) dst[c * G::PM + pos] = __ldg(src + c * P.npts);
  }
}

// Split rate evaluation, first kernel: chemical potential and mobility at
// every point of a 2D/3D field into P.mm, one point per thread, a 32 x 8
// tile of a plane per block.  Same arithmetic as mu_plane64: Laplacian
// neighbour order (operators.py:49-76) +axis0, -axis0, +axis1, -axis1
// (, +axis2, -axis2), then mu = v - lap*kappa (+ s' * l).
//
// Before interpolating, the block orders its points by table cell
// (counting sort on cell_hash), so the lanes of a warp gather the same
// table nodes: a warp-wide corner load then touches one or two cache lines
// instead of one per lane.  Every point is evaluated exactly once (no halo)
// and the order only changes which thread evaluates a point.
template <int DIM, bool VEC, int MINB>
__global__ void __launch_bounds__(256, MINB) k_chem64(RateParams P) {
  constexpr int NT = 256;
  __shared__ double io[2 * S + 1][NT];   // inputs of each point: x, lap, s'
  __shared__ int hist[NT];
  __shared__ int wsum[NT / 32 + 1];
  __shared__ unsigned short order[NT];
  pdl_wait();
  if (P.st->halt) return;
  const int tid = threadIdx.y * 32 + threadIdx.x;
  const int x = blockIdx.x * 32 + threadIdx.x;
  const int y = blockIdx.y * 8 + threadIdx.y;
  const int z = blockIdx.z;
  const bool valid = x < P.nx && y < P.ny;
  const int64_t plane = (int64_t)P.ny * P.nx;
  const int64_t zo = (int64_t)z * plane;
  const int64_t g = zo + (int64_t)y * P.nx + x;
  hist[tid] = 0;
  int key = 0, rank = 0;
  __syncthreads();
  if (valid) {
    auto ld = [&](int64_t gi, double v[S]) {
      const double2 a = __ldg(reinterpret_cast<const double2 *>(P.X + 4 * gi));
      const double2 b = __ldg(reinterpret_cast<const double2 *>(P.X + 4 * gi) + 1);
      v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
    };
    const int xp = x + 1 == P.nx ? 0 : x + 1, xm = x == 0 ? P.nx - 1 : x - 1;
    const int yp = y + 1 == P.ny ? 0 : y + 1, ym = y == 0 ? P.ny - 1 : y - 1;
    double xc[S], lap[S], n0[S], n1[S];
    ld(g, xc);
    if (DIM == 1) {
#pragma unroll
      for (int c = 0; c < S; ++c) lap[c] = 0.0;
    } else if (DIM == 3) {
      const int zp = z + 1 == P.nz ? 0 : z + 1, zm = z == 0 ? P.nz - 1 : z - 1;
      ld((int64_t)zp * plane + (int64_t)y * P.nx + x, n0);
      ld((int64_t)zm * plane + (int64_t)y * P.nx + x, n1);
#pragma unroll
      for (int c = 0; c < S; ++c) lap[c] = n0[c] + n1[c];
      ld(zo + (int64_t)yp * P.nx + x, n0);
      ld(zo + (int64_t)ym * P.nx + x, n1);
#pragma unroll
      for (int c = 0; c < S; ++c) lap[c] = (lap[c] + n0[c]) + n1[c];
    } else {
      ld(zo + (int64_t)yp * P.nx + x, n0);
      ld(zo + (int64_t)ym * P.nx + x, n1);
#pragma unroll
      for (int c = 0; c < S; ++c) lap[c] = n0[c] + n1[c];
    }
    ld(zo + (int64_t)y * P.nx + xp, n0);
    ld(zo + (int64_t)y * P.nx + xm, n1);
#pragma unroll
    for (int c = 0; c < S; ++c) {
      if (DIM == 1)
        lap[c] = ((n0[c] + n1[c]) - 2.0 * xc[c]) * P.inv_dx2;
      else
        lap[c] = (((lap[c] + n0[c]) + n1[c]) - (DIM == 3 ? 6.0 : 4.0) * xc[c]) * P.inv_dx2;
      io[c][tid] = xc[c];
      io[S + c][tid] = lap[c];
    }
    io[2 * S][tid] = P.sp ? __ldg(P.sp + g) : 0.0;
    key = cell_hash(xc, (float)P.T.inv_step);
    rank = atomicAdd(&hist[key], 1);
  }
  __syncthreads();
  const int count = block_exclusive_scan<NT, NT>(hist, wsum, tid);
  if (valid) order[hist[key] + rank] = (unsigned short)tid;
  __syncthreads();
  unsigned flags = 0;
  double v[NP];
  if (tid < count) {
    const int q = order[tid];
    double xq[S], lq[S];
#pragma unroll
    for (int c = 0; c < S; ++c) {
      xq[c] = io[c][q];
      lq[c] = io[S + c][q];
    }
    const double spv = io[2 * S][q];
    const int o[S] = {0, 0, 0, 0};
    interp_win64<VEC>(P.T, xq, nullptr, o, v, &flags);
    // point q of the tile: row q / 32, column q % 32
    const int64_t gq = zo + (int64_t)(blockIdx.y * 8 + (q >> 5)) * P.nx + blockIdx.x * 32 + (q & 31);
#pragma unroll
    for (int c = 0; c < S; ++c) {
      const double lk = lq[c] * P.kappa.v[c];
      double m = v[c] - lk;
      if (P.sp) m = m + spv * P.lvec.v[c];
      P.mm[c * P.npts + gq] = m;
    }
#pragma unroll
    for (int c = 0; c < NM; ++c) P.mm[(S + c) * P.npts + gq] = v[S + c];
  }
  raise_rate_flags(P.st, flags);
}

// Split rate evaluation, first kernel, staged form (VEC tables, 2D/3D): the
// values of k_chem64 bit for bit, with each thread's results put back in
// the shared input rows at its point's tile position, so the mu/M rows of
// P.mm are written in tile order (coalesced) rather than in the table-cell
// order the gathers run in.
template <int DIM, int MINB>
__global__ void __launch_bounds__(256, MINB) k_chem64s(RateParams P) {
  constexpr int NT = 256;
  static_assert(DIM >= 2, "plane tiles");
  __shared__ double io[2 * S + 1][NT];   // inputs of each point (x, lap, s'), then its mu/M
  __shared__ int hist[NT];
  __shared__ int wsum[NT / 32 + 1];
  __shared__ unsigned short order[NT];
  pdl_wait();
  if (P.st->halt) return;
  const int tid = threadIdx.y * 32 + threadIdx.x;
  const int x = blockIdx.x * 32 + threadIdx.x;
  const int y = blockIdx.y * 8 + threadIdx.y;
  const int z = blockIdx.z;
  const bool valid = x < P.nx && y < P.ny;
  const int64_t plane = (int64_t)P.ny * P.nx;
  const int64_t zo = (int64_t)z * plane;
  const int64_t g = zo + (int64_t)y * P.nx + x;
  hist[tid] = 0;
  int key = 0, rank = 0;
  __syncthreads();
  if (valid) {
    auto ld = [&](int64_t gi, double v[S]) {
      const double2 a = __ldg(reinterpret_cast<const double2 *>(P.X + 4 * gi));
      const double2 b = __ldg(reinterpret_cast<const double2 *>(P.X + 4 * gi) + 1);
      v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
    };
    const int xp = x + 1 == P.nx ? 0 : x + 1, xm = x == 0 ? P.nx - 1 : x - 1;
    const int yp = y + 1 == P.ny ? 0 : y + 1, ym = y == 0 ? P.ny - 1 : y - 1;
    double xc[S], lap[S], n0[S], n1[S];
    ld(g, xc);
    if (DIM == 3) {
      const int zp = z + 1 == P.nz ? 0 : z + 1, zm = z == 0 ? P.nz - 1 : z - 1;
      ld((int64_t)zp * plane + (int64_t)y * P.nx + x, n0);
      ld((int64_t)zm * plane + (int64_t)y * P.nx + x, n1);
#pragma unroll
      for (int c = 0; c < S; ++c) lap[c] = n0[c] + n1[c];
      ld(zo + (int64_t)yp * P.nx + x, n0);
      ld(zo + (int64_t)ym * P.nx + x, n1);
#pragma unroll
      for (int c = 0; c < S; ++c) lap[c] = (lap[c] + n0[c]) + n1[c];
    } else {
      ld(zo + (int64_t)yp * P.nx + x, n0);
      ld(zo + (int64_t)ym * P.nx + x, n1);
#pragma unroll
      for (int c = 0; c < S; ++c) lap[c] = n0[c] + n1[c];
    }
    ld(zo + (int64_t)y * P.nx + xp, n0);
    ld(zo + (int64_t)y * P.nx + xm, n1);
#pragma unroll
    for (int c = 0; c < S; ++c) {
      lap[c] = (((lap[c] + n0[c]) + n1[c]) - (DIM == 3 ? 6.0 : 4.0) * xc[c]) * P.inv_dx2;
      io[c][tid] = xc[c];
      io[S + c][tid] = lap[c];
    }
    io[2 * S][tid] = P.sp ? __ldg(P.sp + g) : 0.0;
    key = cell_hash(xc, (float)P.T.inv_step);
    rank = atomicAdd(&hist[key], 1);
  }
  __syncthreads();
  const int count = block_exclusive_scan<NT, NT>(hist, wsum, tid);
  if (valid) order[hist[key] + rank] = (unsigned short)tid;
  __syncthreads();
  unsigned flags = 0;
  if (tid < count) {
    const int q = order[tid];
    double xq[S], lq[S], v[NP];
#pragma unroll
    for (int c = 0; c < S; ++c) {
      xq[c] = io[c][q];
      lq[c] = io[S + c][q];
    }
    const double spv = io[2 * S][q];
    const int o[S] = {0, 0, 0, 0};
    interp_win64<true>(P.T, xq, nullptr, o, v, &flags);
    // column q is this thread's alone: its inputs are read, now its results
#pragma unroll
    for (int c = 0; c < S; ++c) {
      const double lk = lq[c] * P.kappa.v[c];
      double m = v[c] - lk;
      if (P.sp) m = m + spv * P.lvec.v[c];
      io[c][q] = m;
    }
#pragma unroll
    for (int c = 0; c < NM; ++c) io[S + c][q] = v[S + c];
  }
  raise_rate_flags(P.st, flags);
  __syncthreads();
  if (valid) {
#pragma unroll
    for (int r = 0; r < NP; ++r) P.mm[r * P.npts + g] = io[r][tid];
  }
}

// Split rate evaluation, first kernel, shared-gather form: the same values
// as k_chem64 (bit for bit), with the table gathers of up to K points of one
// table cell shared.  A block of 256 threads takes a brick of 256 K points
// (32 x 8 x K in 3D, 32 x 8K in 2D, 256K in 1D):
//   1. per point: x, the Laplacian (k_chem64's order) and s', the table
//      cell (axis_coord of interpolation.py:110-121) or "nearest row";
//   2. counting sort of the points by a hash of their cell (bin 255: points
//      outside the linear region);
//   3. each linear bin's run is cut into work items of up to K points;
//   4. a thread evaluates an item: each corner node is loaded once and its
//      term w * v accumulated into every point of the item, each point with
//      its own weight ((w0 w1) w2) w3 and the reference's left-to-right
//      16-term sum, so every value is the one k_chem64 computes.  Points
//      whose cell differs from the item's first (hash collisions) are set
//      aside;
//   5. the points set aside and the nearest-row points, one per thread;
//   6. coalesced stores of the SoA rows.
constexpr int kChem64Threads = 256;
// Doubles per point of k_chem64i's shared staging, point-major (80 bytes, so
// a point's values move as 16-byte vectors without bank conflicts between
// neighbouring points): x (4), lap (4), s' -- overwritten by mu (4), M (5).
constexpr int kIo64 = 10;

template <int DIM, int K>
struct Chem64Geom {
  static constexpr int NPB = kChem64Threads * K;
  static constexpr int BX = DIM == 1 ? NPB : 32;
  static constexpr int BY = DIM == 1 ? 1 : (DIM == 2 ? 8 * K : 8);
  static constexpr int BZ = DIM == 3 ? K : 1;
  static constexpr int NITEMS = NPB / K + 256;
  // io[kIo64 * NPB] doubles (point-major), cell[NPB] int, items[NITEMS] u32,
  // order/prank/left [NPB] u16, skey/pkey [NPB] u8, hist/cnt/ibase [256] int,
  // wsum + nleft
  static constexpr size_t smem = (size_t)10 * NPB * 8 + NPB * 4 + NITEMS * 4 + 3 * NPB * 2 +
                                 2 * NPB + 3 * 256 * 4 + 16 * 4;
};

template <int DIM, bool VEC, int K, int MINB>
__global__ void __launch_bounds__(kChem64Threads, MINB) k_chem64i(RateParams P) {
  using G = Chem64Geom<DIM, K>;
  constexpr int NT = kChem64Threads, NPB = G::NPB;
  extern __shared__ double2 smd[];
  double *io = reinterpret_cast<double *>(smd);             // kIo64 per point, point-major
  int *cellv = reinterpret_cast<int *>(io + kIo64 * NPB);
  unsigned *items = reinterpret_cast<unsigned *>(cellv + NPB);
  unsigned short *order = reinterpret_cast<unsigned short *>(items + G::NITEMS);
  unsigned short *prank = order + NPB;
  unsigned short *left = prank + NPB;
  unsigned char *skey = reinterpret_cast<unsigned char *>(left + NPB);
  unsigned char *pkey = skey + NPB;
  int *hist = reinterpret_cast<int *>(pkey + NPB);
  int *cnt = hist + 256;
  int *ibase = cnt + 256;
  int *wsum = ibase + 256;
  int *nleft = wsum + 12;
  pdl_wait();
  if (P.st->halt) return;
  const int tid = threadIdx.x;
  const Table &T = P.T;
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
    prank[q] = kNoRank;
    if (x >= P.nx || y >= P.ny || z >= P.nz) continue;
    const int64_t zo = (int64_t)z * plane, g = zo + (int64_t)y * P.nx + x;
    auto ld = [&](int64_t gi, double v[S]) {
      const double2 a = __ldg(reinterpret_cast<const double2 *>(P.X + 4 * gi));
      const double2 b = __ldg(reinterpret_cast<const double2 *>(P.X + 4 * gi) + 1);
      v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
    };
    const int xp = x + 1 == P.nx ? 0 : x + 1, xm = x == 0 ? P.nx - 1 : x - 1;
    double xc[S], lap[S], n0[S], n1[S];
    ld(g, xc);
    if (DIM == 3) {
      const int zp = z + 1 == P.nz ? 0 : z + 1, zm = z == 0 ? P.nz - 1 : z - 1;
      ld((int64_t)zp * plane + (int64_t)y * P.nx + x, n0);
      ld((int64_t)zm * plane + (int64_t)y * P.nx + x, n1);
#pragma unroll
      for (int c = 0; c < S; ++c) lap[c] = n0[c] + n1[c];
    }
    if (DIM >= 2) {
      const int yp = y + 1 == P.ny ? 0 : y + 1, ym = y == 0 ? P.ny - 1 : y - 1;
      ld(zo + (int64_t)yp * P.nx + x, n0);
      ld(zo + (int64_t)ym * P.nx + x, n1);
#pragma unroll
      for (int c = 0; c < S; ++c) lap[c] = DIM == 3 ? (lap[c] + n0[c]) + n1[c] : n0[c] + n1[c];
    }
    ld(zo + (int64_t)y * P.nx + xp, n0);
    ld(zo + (int64_t)y * P.nx + xm, n1);
#pragma unroll
    for (int c = 0; c < S; ++c) {
      if (DIM == 1)
        lap[c] = ((n0[c] + n1[c]) - 2.0 * xc[c]) * P.inv_dx2;
      else
        lap[c] = (((lap[c] + n0[c]) + n1[c]) - (DIM == 3 ? 6.0 : 4.0) * xc[c]) * P.inv_dx2;
      io[q * kIo64 + c] = xc[c];
      io[q * kIo64 + S + c] = lap[c];
    }
    io[q * kIo64 + 8] = P.sp ? __ldg(P.sp + g) : 0.0;
    int ii[S];
    double tt[S];
    int cell = -1, key = 255;
    if (cell64(T, xc, ii, tt)) {
      cell = ((ii[0] * T.n + ii[1]) * T.n + ii[2]) * T.n + ii[3];
      key = (int)((unsigned)(41 * ii[0] + 13 * ii[1] + 5 * ii[2] + ii[3]) % 255u);
    }
    cellv[q] = cell;
    pkey[q] = (unsigned char)key;
    prank[q] = (unsigned short)atomicAdd(&hist[key], 1);
  }
  __syncthreads();
  // 2. counting sort by cell key
  cnt[tid] = hist[tid];
  const int nvalid = block_exclusive_scan<256, NT>(hist, wsum, tid);
  for (int q = tid; q < NPB; q += NT) {
    if (prank[q] == kNoRank) continue;
    const int b = pkey[q], s = hist[b] + prank[q];
    order[s] = (unsigned short)q;
    skey[s] = (unsigned char)b;
  }
  // 3. work items of up to K points of one linear bin
  ibase[tid] = tid == 255 ? 0 : (cnt[tid] + K - 1) / K;
  const int nitems = block_exclusive_scan<256, NT>(ibase, wsum, tid);
  const int lin_end = nvalid - cnt[255];
  for (int s = tid; s < lin_end; s += NT) {
    const int b = skey[s], r = s - hist[b];
    if (r % K == 0) items[ibase[b] + r / K] = (unsigned)s | ((unsigned)min(K, cnt[b] - r) << 16);
  }
  __syncthreads();
  // 4. the work items
  const int64_t s3 = T.stride, s2 = (int64_t)T.n * s3, s1 = (int64_t)T.n * s2,
                s0 = (int64_t)T.n * s1;
  for (int it = tid; it < nitems; it += NT) {
    const unsigned e = items[it];
    const int s = (int)(e & 0xFFFFu), m = (int)(e >> 16);
    int q[K];
    bool use[K];
    double tt[K][S], qq[K][S];
    int cell0 = 0;
#pragma unroll
    for (int j = 0; j < K; ++j) {
      q[j] = j < m ? (int)order[s + j] : 0;
      const int cj = cellv[q[j]];
      if (j == 0) cell0 = cj;
      use[j] = j < m && cj == cell0;
      if (j < m && !use[j]) left[atomicAdd(nleft, 1)] = (unsigned short)q[j];
#pragma unroll
      for (int a = 0; a < S; ++a) {
        int i;
        axis_coord(io[q[j] * kIo64 + a] * T.inv_step, T.n, i, tt[j][a]);
        qq[j][a] = 1.0 - tt[j][a];
      }
    }
    double acc[K][NP];
    const double *base = T.grid + (int64_t)cell0 * s3;
#pragma unroll
    for (int c = 0; c < 16; ++c) {
      const int b0 = (c >> 3) & 1, b1 = (c >> 2) & 1, b2 = (c >> 1) & 1, b3 = c & 1;
      const double *node = base + b0 * s0 + b1 * s1 + b2 * s2 + b3 * s3;
      double v[NP + 1];
      if (VEC) {
        const double2 *n2 = reinterpret_cast<const double2 *>(node);
#pragma unroll
        for (int k = 0; k < (NP + 1) / 2; ++k) {
          const double2 a = __ldg(n2 + k);
          v[2 * k] = a.x;
          v[2 * k + 1] = a.y;
        }
      } else {
#pragma unroll
        for (int p = 0; p < NP; ++p) v[p] = __ldg(node + p);
      }
#pragma unroll
      for (int j = 0; j < K; ++j) {
        const double w = (b0 ? tt[j][0] : qq[j][0]) * (b1 ? tt[j][1] : qq[j][1]) *
                         (b2 ? tt[j][2] : qq[j][2]) * (b3 ? tt[j][3] : qq[j][3]);
#pragma unroll
        for (int p = 0; p < NP; ++p) {
          const double term = w * v[p];
          acc[j][p] = (c == 0) ? term : acc[j][p] + term;
        }
      }
    }
#pragma unroll
    for (int j = 0; j < K; ++j) {
      if (!use[j]) continue;
#pragma unroll
      for (int c = 0; c < S; ++c) {
        const double lk = io[q[j] * kIo64 + S + c] * P.kappa.v[c];
        double mu = acc[j][c] - lk;
        if (P.sp) mu = mu + io[q[j] * kIo64 + 8] * P.lvec.v[c];
        io[q[j] * kIo64 + c] = mu;
      }
#pragma unroll
      for (int c = 0; c < NM; ++c) io[q[j] * kIo64 + S + c] = acc[j][S + c];
    }
  }
  __syncthreads();
  // 5. points set aside and points outside the linear region, one per thread
  unsigned flags = 0;
  const int nnn = cnt[255], nl = nnn + *nleft;
  for (int l = tid; l < nl; l += NT) {
    const int q = l < nnn ? (int)order[lin_end + l] : (int)left[l - nnn];
    double xq[S], v[NP];
#pragma unroll
    for (int c = 0; c < S; ++c) xq[c] = io[q * kIo64 + c];
    const int o[S] = {0, 0, 0, 0};
    interp_win64<VEC>(T, xq, nullptr, o, v, &flags);
#pragma unroll
    for (int c = 0; c < S; ++c) {
      const double lk = io[q * kIo64 + S + c] * P.kappa.v[c];
      double mu = v[c] - lk;
      if (P.sp) mu = mu + io[q * kIo64 + 8] * P.lvec.v[c];
      io[q * kIo64 + c] = mu;
    }
#pragma unroll
    for (int c = 0; c < NM; ++c) io[q * kIo64 + S + c] = v[S + c];
  }
  raise_rate_flags(P.st, flags);
  __syncthreads();
  // 6. coalesced stores of the SoA rows
#pragma unroll 1
  for (int j = 0; j < K; ++j) {
    const int q = tid + j * NT;
    const int qx = q % G::BX, qy = (q / G::BX) % G::BY, qz = q / (G::BX * G::BY);
    const int x = blockIdx.x * G::BX + qx, y = blockIdx.y * G::BY + qy, z = blockIdx.z * G::BZ + qz;
    if (x >= P.nx || y >= P.ny || z >= P.nz) continue;
    const int64_t g = (int64_t)z * plane + (int64_t)y * P.nx + x;
#pragma unroll
    for (int c = 0; c < NP; ++c) P.mm[c * P.npts + g] = io[q * kIo64 + c];
  }
}

// Fold this thread's max |dX/dt| into the block and store the block's max
// in its own slot of P.partial (a plain store: no same-address atomics, no
// fences); k_dt_finish reduces the slots and runs the dt controller.
__device__ __forceinline__ void finish_rate(const RateParams &P, double m, double *red) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  const int tid = threadIdx.y * blockDim.x + threadIdx.x;
  const int nw = (blockDim.x * blockDim.y + 31) >> 5;
  __syncthreads();
  if ((tid & 31) == 0) red[tid >> 5] = m;
  __syncthreads();
  if (tid == 0) {
    for (int w = 1; w < nw; ++w) m = fmax(m, red[w]);
    P.partial[(blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x] = m;
  }
}

// After a rate launch of `nparts` blocks: max |dX/dt| over the block slots,
// then the adaptive-dt rule (system.py:90-112) and dt / time / step on the
// device.  One block.
constexpr int kDtThreads = 1024;
__global__ void __launch_bounds__(kDtThreads) k_dt_finish(RateParams P, int nparts) {
  __shared__ double red[kDtThreads / 32];
  pdl_wait();
  StepState *st = P.st;
  if (st->halt) return;
  double m = 0.0;
  for (int i = threadIdx.x; i < nparts; i += kDtThreads) m = fmax(m, P.partial[i]);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < kDtThreads / 32; ++w) m = fmax(m, red[w]);
    double dt = st->dt;
    if (P.adaptive) dt = adaptive_dt(dt, m, P.ctld, P.t_cfl, P.lower, P.upper, P.factor);
    st->dt = dt;
    st->time = st->time + dt;
    st->xdotmax = m;
    st->step = st->step + 1;
  }
}

// Flux through the face between (X plane XL, pos pl ; mu/M plane ML, pos ql)
// and (XH, ph ; MH, qh), lower -> upper along one axis.
template <int PX, int PM>
__device__ __forceinline__ void face_between(const double *XL, const double *ML, int pl, int ql,
                                             const double *XH, const double *MH, int ph, int qh,
                                             double inv_dx, double J[S]) {
  double Xc[S], Xn[S], Mc[NM], Mn[NM], g[S];
#pragma unroll
  for (int c = 0; c < S; ++c) {
    Xc[c] = XL[c * PX + pl];
    Xn[c] = XH[c * PX + ph];
    g[c] = (MH[c * PM + qh] - ML[c * PM + ql]) * inv_dx;
  }
#pragma unroll
  for (int c = 0; c < NM; ++c) {
    Mc[c] = ML[(S + c) * PM + ql];
    Mn[c] = MH[(S + c) * PM + qh];
  }
  face_flux(Xc, Mc, Xn, Mn, g, J);
}

// All x- and y-faces of one plane tile into Fx / Fy (flat loop: every
// thread takes faces in turn).
template <int TX, int TY, int NTH = TX * TY>
__device__ __forceinline__ void plane_faces(const double *Xp, const double *Mp, double *Fx,
                                            double *Fy, double inv_dx, int tid) {
  using G = PlaneGeom<TX, TY, NTH>;
  for (int f = tid; f < G::NFX + G::NFY; f += G::NT) {
    double J[S];
    if (f < G::NFX) {
      const int fy = f / (TX + 1), fx = f - fy * (TX + 1);
      const int pl = (fy + 2) * G::HX + (fx + 1), ql = (fy + 1) * G::MX + fx;
      face_between<G::PX, G::PM>(Xp, Mp, pl, ql, Xp, Mp, pl + 1, ql + 1, inv_dx, J);
#pragma unroll
      for (int c = 0; c < S; ++c) Fx[c * G::NFX + f] = J[c];
    } else {
      const int f2 = f - G::NFX;
      const int fy = f2 / TX, fx = f2 - fy * TX;
      const int pl = (fy + 1) * G::HX + (fx + 2), ql = fy * G::MX + (fx + 1);
      face_between<G::PX, G::PM>(Xp, Mp, pl, ql, Xp, Mp, pl + G::HX, ql + G::MX, inv_dx, J);
#pragma unroll
      for (int c = 0; c < S; ++c) Fy[c * G::NFY + f2] = J[c];
    }
  }
}

// Stage one X plane (tile + 2-cell halo) into SoA shared memory.
template <int TX, int TY, int NTH = TX * TY>
__device__ __forceinline__ void load_plane(const double *__restrict__ X, int64_t plane_off,
                                           const int *wx, const int *wy, int nx, double *dst,
                                           int tid) {
  using G = PlaneGeom<TX, TY, NTH>;
  for (int pos = tid; pos < G::PX; pos += G::NT) {
    const int hy = pos / G::HX, hx = pos - hy * G::HX;
    const int64_t g = plane_off + (int64_t)wy[hy] * nx + wx[hx];
    const double2 a = __ldg(reinterpret_cast<const double2 *>(X + 4 * g));
    const double2 b = __ldg(reinterpret_cast<const double2 *>(X + 4 * g) + 1);
    dst[0 * G::PX + pos] = a.x;
    dst[1 * G::PX + pos] = a.y;
    dst[2 * G::PX + pos] = b.x;
    dst[3 * G::PX + pos] = b.y;
  }
}

// ------------------------------------------------------------------------
// 2D kernel: one plane tile per block, one point per thread.
// ------------------------------------------------------------------------
// Axis 0 of the (n0, n1) field is the tile's y, axis 1 its x.  Laplacian
// (operators.py:49-60) and divergence (fluxes.py:349) keep the reference's
// axis order: axis-0 terms first.
// A block is NTH threads in one dimension (at least one per tile point; with
// NTH >= the mu/M position count every position takes one pass).  SORT:
// mu/M positions evaluated in table-cell order.
template <int TX, int TY, int MINB, bool VEC, bool WIN, bool SPLIT = false, int NTH = TX * TY,
          int SORT = 0, bool PERPOINT = false>
__global__ void __launch_bounds__(NTH, MINB) k_rate_tile2d(RateParams P) {
  using G = PlaneGeom<TX, TY, NTH>;
  static_assert(NTH >= TX * TY && NTH % 32 == 0, "one thread per tile point at least");
  pdl_wait();
  if (P.st->halt) return;
  extern __shared__ double sm[];
  double *Xs = sm;                       // [S][PX]
  double *Ms = Xs + S * G::PX;           // [NP][PM]
  double *Fx = Ms + NP * G::PM;          // [S][NFX]
  double *Fy = Fx + S * G::NFX;          // [S][NFY]   (Fx/Fy also hold the table window)
  double *red = Fy + S * G::NFY;         // [NT/32]
  int *wx = reinterpret_cast<int *>(red + G::NT / 32);   // [HX]
  int *wy = wx + G::HX;                                  // [HY]
  int *win_lo = wy + G::HY;                              // [S+1] window origin, valid
  SortScratch ss{};
  if constexpr (SORT) {
    ss.hist = win_lo + S + 1;                            // [256]
    ss.wsum = ss.hist + 256;                             // [NT/32 + 1]
    ss.order = reinterpret_cast<unsigned short *>(ss.wsum + G::NT / 32 + 1);   // [PM]
    ss.rank = ss.order + G::PM;                          // [PM]
    ss.key = reinterpret_cast<unsigned char *>(ss.rank + G::PM);               // [PM]
  }
  const int tid = threadIdx.x, tx = tid % TX, ty = tid / TX;
  const int x0 = blockIdx.x * TX, y0 = blockIdx.y * TY;
  unsigned flags = 0;
  if (tid == 0) win_lo[S] = 0;

  for (int i = tid; i < G::HX + G::HY; i += G::NT) {
    if (i < G::HX) wx[i] = wrap_any(x0 + i - 2, P.nx);
    else wy[i - G::HX] = wrap_any(y0 + (i - G::HX) - 2, P.ny);
  }
  __syncthreads();
  load_plane<TX, TY, NTH>(P.X, 0, wx, wy, P.nx, Xs, tid);
  __syncthreads();
  if constexpr (SPLIT)
    load_mu_plane<TX, TY, NTH>(P, 0, wx, wy, false, Ms, tid);
  else
    mu_plane64<TX, TY, 2, VEC, WIN, NTH, SORT>(P, nullptr, Xs, nullptr, Ms, 0, wx, wy, false,
                                               reinterpret_cast<double2 *>(Fx), win_lo, &flags,
                                               tid, ss);
  __syncthreads();
  double jyp[S], jym[S], jxp[S], jxm[S];
  const bool mine = tid < TX * TY && x0 + tx < P.nx && y0 + ty < P.ny;
  if constexpr (PERPOINT) {
    // each point evaluates its four faces from the shared planes (each face
    // by both of its cells, with identical operands and operation order)
    if (mine) {
      const int pX = (ty + 2) * G::HX + (tx + 2), pM = (ty + 1) * G::MX + (tx + 1);
      face_between<G::PX, G::PM>(Xs, Ms, pX, pM, Xs, Ms, pX + G::HX, pM + G::MX, P.inv_dx, jyp);
      face_between<G::PX, G::PM>(Xs, Ms, pX - G::HX, pM - G::MX, Xs, Ms, pX, pM, P.inv_dx, jym);
      face_between<G::PX, G::PM>(Xs, Ms, pX, pM, Xs, Ms, pX + 1, pM + 1, P.inv_dx, jxp);
      face_between<G::PX, G::PM>(Xs, Ms, pX - 1, pM - 1, Xs, Ms, pX, pM, P.inv_dx, jxm);
    }
  } else {
    plane_faces<TX, TY, NTH>(Xs, Ms, Fx, Fy, P.inv_dx, tid);
    __syncthreads();
    if (mine) {
#pragma unroll
      for (int c = 0; c < S; ++c) {
        jyp[c] = Fy[c * G::NFY + (ty + 1) * TX + tx];
        jym[c] = Fy[c * G::NFY + ty * TX + tx];
        jxp[c] = Fx[c * G::NFX + ty * (TX + 1) + tx + 1];
        jxm[c] = Fx[c * G::NFX + ty * (TX + 1) + tx];
      }
    }
  }
  double vmax = 0.0;
  if (mine) {
    double out[S];
#pragma unroll
    for (int c = 0; c < S; ++c) {
      double a = jyp[c] - jym[c];
      a = a + jxp[c];
      a = a - jxm[c];
      out[c] = a * P.inv_dx;
      const double v = fabs(out[c]);
      if (v > vmax) vmax = v;
    }
    const int64_t g = (int64_t)(y0 + ty) * P.nx + (x0 + tx);
    double2 *o = reinterpret_cast<double2 *>(P.dX + 4 * g);
    o[0] = make_double2(out[0], out[1]);
    o[1] = make_double2(out[2], out[3]);
  }
  raise_rate_flags(P.st, flags);
  finish_rate(P, vmax, red);
}

template <int TX, int TY, int NTH = TX * TY, int SORT = 0>
constexpr size_t tile2d_smem() {
  using G = PlaneGeom<TX, TY, NTH>;
  static_assert(S * (G::NFX + G::NFY) * sizeof(double) >= kWinNodes64 * kNodeV64 * sizeof(double2),
                "face buffers must hold the table window");
  const size_t sort = SORT ? (256 + G::NT / 32 + 1) * sizeof(int) + G::PM * (2 * 2 + 1) : 0;
  return (S * G::PX + NP * G::PM + S * G::NFX + S * G::NFY + G::NT / 32) * sizeof(double) +
         (G::HX + G::HY + S + 1) * sizeof(int) + sort;
}

// ------------------------------------------------------------------------
// 3D kernel: plane tile marching along axis 0
// ------------------------------------------------------------------------
// Each block owns a TY x TX tile of (axis 1, axis 2) and a chunk of axis-0
// planes.  Rings in shared memory: 3 X planes (2-cell halo), 2 mu/M planes
// (1-cell halo); a persistent table window.  Per output plane z: stage
// X(z+2), evaluate mu/M(z+1), each point's +z face, then the y-faces and
// the x-faces through one face buffer, forming the divergence in the
// reference's axis order: (+z - -z) + (+y - -y) + (+x - -x), with the -z
// face kept in registers from plane z-1.  Laplacian order
// (operators.py:68-76): +z, -z, +y, -y, +x, -x.

// One family of faces of a plane tile into F: AXIS 0 = x-faces (TY x (TX+1)),
// AXIS 1 = y-faces ((TY+1) x TX).
template <int TX, int TY, int AXIS>
__device__ __forceinline__ void plane_faces_axis(const double *Xp, const double *Mp, double *F,
                                                 double inv_dx, int tid) {
  using G = PlaneGeom<TX, TY>;
  constexpr int NF = AXIS == 0 ? G::NFX : G::NFY;
  for (int f = tid; f < NF; f += G::NT) {
    double J[S];
    if (AXIS == 0) {
      const int fy = f / (TX + 1), fx = f - fy * (TX + 1);
      const int pl = (fy + 2) * G::HX + (fx + 1), ql = (fy + 1) * G::MX + fx;
      face_between<G::PX, G::PM>(Xp, Mp, pl, ql, Xp, Mp, pl + 1, ql + 1, inv_dx, J);
    } else {
      const int fy = f / TX, fx = f - fy * TX;
      const int pl = (fy + 1) * G::HX + (fx + 2), ql = fy * G::MX + (fx + 1);
      face_between<G::PX, G::PM>(Xp, Mp, pl, ql, Xp, Mp, pl + G::HX, ql + G::MX, inv_dx, J);
    }
#pragma unroll
    for (int c = 0; c < S; ++c) F[c * NF + f] = J[c];
  }
}

template <int TX, int TY>
struct March64Geom {
  using G = PlaneGeom<TX, TY>;
  static constexpr int NFMAX = G::NFX > G::NFY ? G::NFX : G::NFY;
};

template <int TX, int TY, int MINB, bool VEC, bool WIN, bool SPLIT = false, int SORT = 0,
          bool PERPOINT = false>
__global__ void __launch_bounds__(TX * TY, MINB) k_rate_march3d(RateParams P, int zc) {
  using G = PlaneGeom<TX, TY>;
  pdl_wait();
  if (P.st->halt) return;
  extern __shared__ double sm[];
  double *Xs = sm;                                           // [3][S][PX]
  double *Ms = Xs + 3 * S * G::PX;                           // [2][NP][PM]
  double *F = Ms + 2 * NP * G::PM;                           // [S][NFMAX]
  double2 *win = reinterpret_cast<double2 *>(F + S * March64Geom<TX, TY>::NFMAX);
  double *red = reinterpret_cast<double *>(win + kWinNodes64 * kNodeV64);   // [NT/32]
  int *wx = reinterpret_cast<int *>(red + G::NT / 32);
  int *wy = wx + G::HX;
  int *win_lo = wy + G::HY;                                  // [S+1]
  SortScratch ss{};
  if constexpr (SORT) {
    ss.hist = win_lo + S + 1;                                // [256]
    ss.wsum = ss.hist + 256;                                 // [NT/32 + 1]
    ss.order = reinterpret_cast<unsigned short *>(ss.wsum + G::NT / 32 + 1);   // [PM]
    ss.rank = ss.order + G::PM;                              // [PM]
    ss.key = reinterpret_cast<unsigned char *>(ss.rank + G::PM);               // [PM]
  }
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
  const int x0 = blockIdx.x * TX, y0 = blockIdx.y * TY;
  const int zb = blockIdx.z * zc;
  const int ze = min(zb + zc, P.nz);
  const int64_t plane = (int64_t)P.ny * P.nx;
  unsigned flags = 0;

  for (int i = tid; i < G::HX + G::HY; i += G::NT) {
    if (i < G::HX) wx[i] = wrap_any(x0 + i - 2, P.nx);
    else wy[i - G::HX] = wrap_any(y0 + (i - G::HX) - 2, P.ny);
  }
  if (tid == 0) win_lo[S] = 0;
  auto xplane = [&](int z) { return Xs + ((z - zb + 3) % 3) * S * G::PX; };
  auto mplane = [&](int z) { return Ms + ((z - zb + 2) & 1) * NP * G::PM; };
  auto load_x = [&](int z) {
    load_plane<TX, TY>(P.X, (int64_t)wrap_any(z, P.nz) * plane, wx, wy, P.nx, xplane(z), tid);
  };
  auto compute_mu = [&](int z, bool interior_only) {
    if constexpr (SPLIT)
      load_mu_plane<TX, TY>(P, (int64_t)wrap_any(z, P.nz) * plane, wx, wy, interior_only,
                            mplane(z), tid);
    else
      mu_plane64<TX, TY, 3, VEC, WIN, TX * TY, SORT>(P, xplane(z - 1), xplane(z), xplane(z + 1),
                                                     mplane(z), (int64_t)wrap_any(z, P.nz) * plane,
                                                     wx, wy, interior_only, win, win_lo, &flags,
                                                     tid, ss);
  };
  const int pX = (ty + 2) * G::HX + (tx + 2);
  const int pM = (ty + 1) * G::MX + (tx + 1);
  const bool in_tile = (x0 + tx < P.nx) && (y0 + ty < P.ny);

  __syncthreads();
  if constexpr (SPLIT) {          // faces need X and mu/M of planes z and z+1 only
    load_x(zb - 1);
    load_x(zb);
    compute_mu(zb - 1, true);
    compute_mu(zb, false);
  } else {
    load_x(zb - 2);
    load_x(zb - 1);
    load_x(zb);
    __syncthreads();
    compute_mu(zb - 1, true);
    __syncthreads();
    load_x(zb + 1);
    __syncthreads();
    compute_mu(zb, false);
  }
  __syncthreads();
  double Jm[S];
  face_between<G::PX, G::PM>(xplane(zb - 1), mplane(zb - 1), pX, pM, xplane(zb), mplane(zb), pX,
                             pM, P.inv_dx, Jm);
  double vmax = 0.0;
  for (int z = zb; z < ze; ++z) {
    __syncthreads();
    if constexpr (SPLIT) {
      load_x(z + 1);
      compute_mu(z + 1, false);
    } else {
      load_x(z + 2);
      __syncthreads();
      compute_mu(z + 1, false);
    }
    __syncthreads();
    double a[S];
    face_between<G::PX, G::PM>(xplane(z), mplane(z), pX, pM, xplane(z + 1), mplane(z + 1), pX,
                               pM, P.inv_dx, a);
#pragma unroll
    for (int c = 0; c < S; ++c) {
      const double jz = a[c];
      a[c] = jz - Jm[c];
      Jm[c] = jz;
    }
    if constexpr (PERPOINT) {
      // each point evaluates its four in-plane faces (each face by both of
      // its cells, identical operands and order): no face buffer, no barriers
      if (in_tile) {
        const double *Xp = xplane(z), *Mp = mplane(z);
        double jyp[S], jym[S], jxp[S], jxm[S], out[S];
        face_between<G::PX, G::PM>(Xp, Mp, pX, pM, Xp, Mp, pX + G::HX, pM + G::MX, P.inv_dx, jyp);
        face_between<G::PX, G::PM>(Xp, Mp, pX - G::HX, pM - G::MX, Xp, Mp, pX, pM, P.inv_dx, jym);
        face_between<G::PX, G::PM>(Xp, Mp, pX, pM, Xp, Mp, pX + 1, pM + 1, P.inv_dx, jxp);
        face_between<G::PX, G::PM>(Xp, Mp, pX - 1, pM - 1, Xp, Mp, pX, pM, P.inv_dx, jxm);
#pragma unroll
        for (int c = 0; c < S; ++c) {
          double v = a[c] + jyp[c];
          v = v - jym[c];
          v = v + jxp[c];
          v = v - jxm[c];
          out[c] = v * P.inv_dx;
          const double m = fabs(out[c]);
          if (m > vmax) vmax = m;
        }
        const int64_t g = (int64_t)z * plane + (int64_t)(y0 + ty) * P.nx + (x0 + tx);
        double2 *o = reinterpret_cast<double2 *>(P.dX + 4 * g);
        o[0] = make_double2(out[0], out[1]);
        o[1] = make_double2(out[2], out[3]);
      }
      continue;
    }
    plane_faces_axis<TX, TY, 1>(xplane(z), mplane(z), F, P.inv_dx, tid);
    __syncthreads();
#pragma unroll
    for (int c = 0; c < S; ++c) {
      a[c] = a[c] + F[c * G::NFY + (ty + 1) * TX + tx];
      a[c] = a[c] - F[c * G::NFY + ty * TX + tx];
    }
    __syncthreads();
    plane_faces_axis<TX, TY, 0>(xplane(z), mplane(z), F, P.inv_dx, tid);
    __syncthreads();
    if (in_tile) {
      double out[S];
#pragma unroll
      for (int c = 0; c < S; ++c) {
        double v = a[c] + F[c * G::NFX + ty * (TX + 1) + tx + 1];
        v = v - F[c * G::NFX + ty * (TX + 1) + tx];
        out[c] = v * P.inv_dx;
        const double m = fabs(out[c]);
        if (m > vmax) vmax = m;
      }
      const int64_t g = (int64_t)z * plane + (int64_t)(y0 + ty) * P.nx + (x0 + tx);
      double2 *o = reinterpret_cast<double2 *>(P.dX + 4 * g);
      o[0] = make_double2(out[0], out[1]);
      o[1] = make_double2(out[2], out[3]);
    }
  }
  raise_rate_flags(P.st, flags);
  finish_rate(P, vmax, red);
}

// ------------------------------------------------------------------------
// Split rate evaluation, second kernel in 3D: faces and divergence of a
// TY x TX plane tile marching along axis 0, from X and the mu/M rows that
// k_chem64 wrote.  The X and mu/M of each plane (tile + 1-cell halo) go
// through a three-plane ring in shared memory that cp.async fills two
// planes ahead, so the loads of plane z+2 run under the faces of plane z.
// Faces and the divergence sum in k_rate_march3d's order (fluxes.py:352-395:
// axis 0, then 1, then 2), so the same bits.
// ------------------------------------------------------------------------
template <int TX, int TY>
struct Flux3Geom64 {
  static constexpr int MX = TX + 2, MY = TY + 2, PM = MX * MY, NT = TX * TY;
  static constexpr int NFX = TY * (TX + 1), NFY = (TY + 1) * TX;
  static constexpr size_t slot = (size_t)(S + NP) * PM;          // doubles: X rows, then mu/M rows
  static constexpr size_t smem(bool perpoint) {
    return (3 * slot + (perpoint ? 0 : (size_t)S * (NFX + NFY)) + NT / 32) * sizeof(double) +
           (MX + MY) * sizeof(int);
  }
};

// X, mu and M of one position read out of a plane's rows (stride PM), and
// the face flux between two such positions, lower -> upper: the operands
// and operation order of face_between, so the same bits.
struct Pt64 {
  double x[S], mu[S], m[NM];
};

template <int PM>
__device__ __forceinline__ void load_pt64(const double *X, const double *M, int p, Pt64 &q) {
#pragma unroll
  for (int c = 0; c < S; ++c) {
    q.x[c] = X[c * PM + p];
    q.mu[c] = M[c * PM + p];
  }
#pragma unroll
  for (int c = 0; c < NM; ++c) q.m[c] = M[(S + c) * PM + p];
}

__device__ __forceinline__ void face_pts64(const Pt64 &lo, const Pt64 &hi, double inv_dx,
                                           double J[S]) {
  double g[S];
#pragma unroll
  for (int c = 0; c < S; ++c) g[c] = (hi.mu[c] - lo.mu[c]) * inv_dx;
  face_flux(lo.x, lo.m, hi.x, hi.m, g, J);
}

template <int TX, int TY, int MINB, bool PERPOINT>
__global__ void __launch_bounds__(TX * TY, MINB) k_flux3_64(RateParams P, int zc) {
  using G = Flux3Geom64<TX, TY>;
  pdl_wait();
  if (P.st->halt) return;
  extern __shared__ double sm[];
  double *ring = sm;                                         // [3][S + NP][PM]
  double *Fx = ring + 3 * G::slot;                           // [S][NFX] (flat faces)
  double *Fy = Fx + (PERPOINT ? 0 : S * G::NFX);             // [S][NFY]
  double *red = Fy + (PERPOINT ? 0 : S * G::NFY);            // [NT/32]
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
  auto sX = [&](int z) { return ring + ((z - zb + 3) % 3) * G::slot; };
  auto sM = [&](int z) { return sX(z) + S * G::PM; };
  auto issue = [&](int z, bool interior_only) {
    const int64_t zoff = (int64_t)wrap_any(z, P.nz) * plane;
    double *x = sX(z), *m = sM(z);
    for (int pos = tid; pos < G::PM; pos += G::NT) {
      const int my = pos / G::MX, mx = pos - my * G::MX;
      const bool ex = (mx == 0 || mx == G::MX - 1), ey = (my == 0 || my == G::MY - 1);
      if (interior_only ? (ex || ey) : (ex && ey)) continue;
      const int64_t g = zoff + (int64_t)wy[my] * P.nx + wx[mx];
#pragma unroll
      for (int c = 0; c < S; ++c) __pipeline_memcpy_async(x + c * G::PM + pos, P.X + 4 * g + c, 8);
#pragma unroll
      for (int r = 0; r < NP; ++r)
        __pipeline_memcpy_async(m + r * G::PM + pos, P.mm + r * P.npts + g, 8);
    }
    __pipeline_commit();
  };
  auto face = [&](int zl, int pl, int zh, int ph, double J[S]) {
    face_between<G::PM, G::PM>(sX(zl), sM(zl), pl, pl, sX(zh), sM(zh), ph, ph, P.inv_dx, J);
  };
  const int p = (ty + 1) * G::MX + (tx + 1);
  const bool in_tile = (x0 + tx < P.nx) && (y0 + ty < P.ny);
  issue(zb - 1, true);
  issue(zb, false);
  issue(zb + 1, false);
  __pipeline_wait_prior(1);
  __syncthreads();
  // PERPOINT: this point's X/mu/M at plane z stay in registers (cur) and
  // become the lower side of the next plane's axis-0 face.
  Pt64 cur;
  double Jm[S];
  if constexpr (PERPOINT) {
    Pt64 below;
    load_pt64<G::PM>(sX(zb - 1), sM(zb - 1), p, below);
    load_pt64<G::PM>(sX(zb), sM(zb), p, cur);
    face_pts64(below, cur, P.inv_dx, Jm);
  } else {
    face(zb - 1, p, zb, p, Jm);
  }
  double vmax = 0.0;
  for (int z = zb; z < ze; ++z) {
    __pipeline_wait_prior(0);          // plane z+1 copied (this thread's part)
    __syncthreads();                   // ... and every thread's; the slot of z-1 is free
    if (z + 2 <= ze) issue(z + 2, false);
    double a[S];
    double jyp[S], jym[S], jxp[S], jxm[S];
    if constexpr (PERPOINT) {
      // each point evaluates its four in-plane faces (each face by both of
      // its cells, identical operands and order)
      Pt64 up, nb;
      load_pt64<G::PM>(sX(z + 1), sM(z + 1), p, up);
      face_pts64(cur, up, P.inv_dx, a);
      const double *Xz = sX(z), *Mz = sM(z);
      load_pt64<G::PM>(Xz, Mz, p + G::MX, nb);
      face_pts64(cur, nb, P.inv_dx, jyp);
      load_pt64<G::PM>(Xz, Mz, p - G::MX, nb);
      face_pts64(nb, cur, P.inv_dx, jym);
      load_pt64<G::PM>(Xz, Mz, p + 1, nb);
      face_pts64(cur, nb, P.inv_dx, jxp);
      load_pt64<G::PM>(Xz, Mz, p - 1, nb);
      face_pts64(nb, cur, P.inv_dx, jxm);
      cur = up;
    } else {
      face(z, p, z + 1, p, a);
    }
#pragma unroll
    for (int c = 0; c < S; ++c) {
      const double jz = a[c];
      a[c] = jz - Jm[c];
      Jm[c] = jz;
    }
    if constexpr (!PERPOINT) {
      for (int f = tid; f < G::NFX + G::NFY; f += G::NT) {
        double J[S];
        if (f < G::NFX) {
          const int fy = f / (TX + 1), fx = f - fy * (TX + 1);
          const int pl = (fy + 1) * G::MX + fx;
          face(z, pl, z, pl + 1, J);
#pragma unroll
          for (int c = 0; c < S; ++c) Fx[c * G::NFX + f] = J[c];
        } else {
          const int f2 = f - G::NFX;
          const int fy = f2 / TX, fx = f2 - fy * TX;
          const int pl = fy * G::MX + (fx + 1);
          face(z, pl, z, pl + G::MX, J);
#pragma unroll
          for (int c = 0; c < S; ++c) Fy[c * G::NFY + f2] = J[c];
        }
      }
      __syncthreads();
#pragma unroll
      for (int c = 0; c < S; ++c) {
        jyp[c] = Fy[c * G::NFY + (ty + 1) * TX + tx];
        jym[c] = Fy[c * G::NFY + ty * TX + tx];
        jxp[c] = Fx[c * G::NFX + ty * (TX + 1) + tx + 1];
        jxm[c] = Fx[c * G::NFX + ty * (TX + 1) + tx];
      }
    }
    if (in_tile) {
      double out[S];
#pragma unroll
      for (int c = 0; c < S; ++c) {
        double v = a[c] + jyp[c];
        v = v - jym[c];
        v = v + jxp[c];
        v = v - jxm[c];
        out[c] = v * P.inv_dx;
        const double m = fabs(out[c]);
        if (m > vmax) vmax = m;
      }
      const int64_t g = (int64_t)z * plane + (int64_t)(y0 + ty) * P.nx + (x0 + tx);
      double2 *o = reinterpret_cast<double2 *>(P.dX + 4 * g);
      o[0] = make_double2(out[0], out[1]);
      o[1] = make_double2(out[2], out[3]);
    }
  }
  __pipeline_wait_prior(0);
  finish_rate(P, vmax, red);
}

template <int TX, int TY, int SORT = 0>
constexpr size_t march3d_smem() {
  using G = PlaneGeom<TX, TY>;
  const size_t sort = SORT ? (256 + G::NT / 32 + 1) * sizeof(int) + G::PM * (2 * 2 + 1) : 0;
  return (3 * S * G::PX + 2 * NP * G::PM + S * March64Geom<TX, TY>::NFMAX + G::NT / 32) *
             sizeof(double) +
         kWinNodes64 * kNodeV64 * sizeof(double2) + (G::HX + G::HY + S + 1) * sizeof(int) + sort;
}

// ------------------------------------------------------------------------
// 1D kernel: a tile of TX points with halos, no marching.
// ------------------------------------------------------------------------
template <int TX, bool VEC>
__global__ void __launch_bounds__(TX) k_rate_1d(RateParams P) {
  pdl_wait();
  if (P.st->halt) return;
  constexpr int HX = TX + 4, MX = TX + 2;
  __shared__ double Xs[S][HX];
  __shared__ double Ms[NP][MX];
  __shared__ double Fx[S][TX + 1];
  __shared__ double red[(TX + 31) / 32];
  const int tx = threadIdx.x;
  const int x0 = blockIdx.x * TX;
  const int n = P.nx;
  unsigned flags = 0;
  for (int pos = tx; pos < HX; pos += TX) {
    const int g = wrap_any(x0 + pos - 2, n);
    const double2 a = __ldg(reinterpret_cast<const double2 *>(P.X + 4 * (int64_t)g));
    const double2 b = __ldg(reinterpret_cast<const double2 *>(P.X + 4 * (int64_t)g) + 1);
    Xs[0][pos] = a.x;
    Xs[1][pos] = a.y;
    Xs[2][pos] = b.x;
    Xs[3][pos] = b.y;
  }
  __syncthreads();
  for (int pos = tx; pos < MX; pos += TX) {
    const int px = pos + 1;
    double x[S], lap[S];
#pragma unroll
    for (int c = 0; c < S; ++c) {
      x[c] = Xs[c][px];
      lap[c] = (Xs[c][px + 1] + Xs[c][px - 1] - 2.0 * x[c]) * P.inv_dx2;
    }
    const double spv = P.sp ? __ldg(P.sp + wrap_any(x0 + pos - 1, n)) : 0.0;
    double mu[S], M[NM];
    chem_point<VEC>(P, x, lap, spv, mu, M, &flags);
#pragma unroll
    for (int c = 0; c < S; ++c) Ms[c][pos] = mu[c];
#pragma unroll
    for (int c = 0; c < NM; ++c) Ms[S + c][pos] = M[c];
  }
  __syncthreads();
  // face f lies between mu/M positions f and f+1 (X positions f+1, f+2)
  for (int f = tx; f < TX + 1; f += TX) {
    double Xc[S], Xn[S], Mc[NM], Mn[NM], g[S], J[S];
#pragma unroll
    for (int c = 0; c < S; ++c) {
      Xc[c] = Xs[c][f + 1];
      Xn[c] = Xs[c][f + 2];
      g[c] = (Ms[c][f + 1] - Ms[c][f]) * P.inv_dx;
    }
#pragma unroll
    for (int c = 0; c < NM; ++c) {
      Mc[c] = Ms[S + c][f];
      Mn[c] = Ms[S + c][f + 1];
    }
    face_flux(Xc, Mc, Xn, Mn, g, J);
#pragma unroll
    for (int c = 0; c < S; ++c) Fx[c][f] = J[c];
  }
  __syncthreads();
  double vmax = 0.0;
  if (x0 + tx < n) {
    double out[S];
#pragma unroll
    for (int c = 0; c < S; ++c) {
      out[c] = (Fx[c][tx + 1] - Fx[c][tx]) * P.inv_dx;
      const double v = fabs(out[c]);
      if (v > vmax) vmax = v;
    }
    double2 *o = reinterpret_cast<double2 *>(P.dX + 4 * (int64_t)(x0 + tx));
    o[0] = make_double2(out[0], out[1]);
    o[1] = make_double2(out[2], out[3]);
  }
  raise_rate_flags(P.st, flags);
  finish_rate(P, vmax, red);
}

// ------------------------------------------------------------------------
// Update + clamp + next misfit + out_of_bounds test
// ------------------------------------------------------------------------
struct UpdateParams {
  double *X;
  const double *dX;
  int64_t npts;
  StepState *st;
  Vec4 x0, lvec;
  double *s;            // misfit scalar for the next step, or nullptr
  int oob_interval;
};

// out_of_bounds (phasefield5d/solver/system.py:12-53) flags for one point.
__device__ __forceinline__ unsigned oob_flags(const double x[S]) {
  unsigned f = 0;
  double sum = 0.0;
#pragma unroll
  for (int c = 0; c < S; ++c) {
    if (!isfinite(x[c])) f |= PF5D_FLAG_NONFINITE;
    sum = sum + x[c];
    if (x[c] < 0.0 - 1e-3 || x[c] > 1.0 + 1e-3) f |= PF5D_FLAG_OOB_HARD;
    if (x[c] < 0.0 - 1e-5 || x[c] > 1.0 + 1e-5) f |= PF5D_FLAG_OOB_SOFT;
  }
  if (sum > 1.0 + 1e-3 || sum < 0.0 - 1e-3) f |= PF5D_FLAG_OOB_HARD;
  if (sum > 1.0 + 1e-5 || sum < 0.0 - 1e-5) f |= PF5D_FLAG_OOB_SOFT;
  return f;
}

__device__ __forceinline__ void raise_flags(StepState *st, unsigned f) {
  if (!f) return;
  atomicOr(&st->flags, f);
  if (f & (PF5D_FLAG_NONFINITE | PF5D_FLAG_OOB_HARD)) atomicExch(&st->halt, 1u);
}

__global__ void k_update_step(UpdateParams U) {
  pdl_wait();
  StepState *st = U.st;
  if (st->halt) return;
  const double dt = st->dt;
  const bool check = U.oob_interval > 0 && (st->step % U.oob_interval) == 0;
  unsigned f = 0;
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < U.npts;
       p += (int64_t)gridDim.x * blockDim.x) {
    double2 *xp = reinterpret_cast<double2 *>(U.X + 4 * p);
    const double2 *dp = reinterpret_cast<const double2 *>(U.dX + 4 * p);
    const double2 a = xp[0], b = xp[1], da = dp[0], db = dp[1];
    double x[S] = {a.x, a.y, b.x, b.y};
    const double d[S] = {da.x, da.y, db.x, db.y};
#pragma unroll
    for (int c = 0; c < S; ++c) x[c] = x[c] + d[c] * dt;     // dX *= dt; X += dX
    double total = 0.0;
#pragma unroll
    for (int c = 0; c < S; ++c) total = total + x[c];
    if (total > 1.0) {
      const double inv = 1.0 / total;
#pragma unroll
      for (int c = 0; c < S; ++c) x[c] = x[c] * inv;
    }
    xp[0] = make_double2(x[0], x[1]);
    xp[1] = make_double2(x[2], x[3]);
    if (U.s) {
      double acc = 0.0;
#pragma unroll
      for (int c = 0; c < S; ++c) acc = acc + (x[c] - U.x0.v[c]) * U.lvec.v[c];
      U.s[p] = acc;
    }
    if (check) f |= oob_flags(x);
  }
  raise_flags(st, f);
}

// The step-0 out_of_bounds test on the initial field.
__global__ void k_check_state(const double *X, int64_t npts, StepState *st) {
  unsigned f = 0;
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < npts;
       p += (int64_t)gridDim.x * blockDim.x) {
    double x[S];
#pragma unroll
    for (int c = 0; c < S; ++c) x[c] = X[4 * p + c];
    f |= oob_flags(x);
  }
  raise_flags(st, f);
}

constexpr int kMeanBlocks = 512;

// FP64 per-component sums of X, two passes (deterministic order).
__global__ void k_mean_partial(const double *__restrict__ X, int64_t npts, double *partial) {
  __shared__ double red[S][8];
  double acc[S] = {0.0, 0.0, 0.0, 0.0};
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < npts;
       p += (int64_t)gridDim.x * blockDim.x)
#pragma unroll
    for (int c = 0; c < S; ++c) acc[c] += X[4 * p + c];
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

__global__ void k_mean_final(const double *partial, int nparts, double *out) {
  if (threadIdx.x < S) {
    double v = 0.0;
    for (int b = 0; b < nparts; ++b) v += partial[b * S + threadIdx.x];
    out[threadIdx.x] = v;
  }
}

}  // namespace pf5d

using namespace pf5d;

namespace pf5d {

// The 1D elastic term in closed form, in place: s (the misfit) ->
// s' = bn (s - mean s) + b0 mean s, where bn is B(k) for every k != 0 and
// b0 is B(0).  That is irfft(B rfft(s)) (elastic.py:250-263) exactly, for a
// B(k) that depends on k only through its sign, as every 1D B(k) does.  One
// block: per-thread sums over a fixed stride, then a fixed tree, so the
// mean has the same bits on every run.
constexpr int kElastic1dThreads = 1024;
constexpr int64_t kElastic1dMax = 16384;     // points of a 1D solve that use it
__global__ void __launch_bounds__(kElastic1dThreads)
    k_elastic1d(double *s, int64_t n, double bn, double b0, const unsigned *halt) {
  __shared__ double red[kElastic1dThreads / 32];
  pdl_wait();
  if (*halt) return;
  const int t = threadIdx.x;
  double acc = 0.0;
  for (int64_t i = t; i < n; i += kElastic1dThreads) acc = acc + s[i];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) acc = acc + __shfl_xor_sync(0xffffffffu, acc, o);
  if ((t & 31) == 0) red[t >> 5] = acc;
  __syncthreads();
  double tot = red[0];
  for (int w = 1; w < kElastic1dThreads / 32; ++w) tot = tot + red[w];
  const double mean = tot / (double)n;
  for (int64_t i = t; i < n; i += kElastic1dThreads) s[i] = bn * (s[i] - mean) + b0 * mean;
}

}  // namespace pf5d

struct pf5d_stepper {
  pf5d_stepper_desc d{};
  int64_t shape[3] = {1, 1, 1};
  int64_t npts = 0;
  double *X = nullptr;
  double *dX = nullptr;
  double *s = nullptr;
  cufftDoubleComplex *k = nullptr;
  double *bk = nullptr;
  FFTPair fft;
  StepState *st = nullptr;
  RateParams rp{};
  UpdateParams up{};
  cudaStream_t cap = nullptr;
  std::map<int64_t, cudaGraphExec_t> graphs;
  dim3 rate_grid, rate_block;
  size_t rate_smem = 0;
  int zc = 1;
  bool vec = false;
  int variant = 0;
  Stepper32 *s32 = nullptr;      // FP32C form (all calls delegate)
  double *mass_ws = nullptr;     // FP64 mean reduction workspace
  double *mm = nullptr;          // split-rate mu/M buffer (also save-step diagnostics)
  double *diag_ws = nullptr;     // save-step partial rows + mean
  double *partial = nullptr;     // rate kernel block maxima
  bool closed1d = false;         // 1D elastic term in closed form (k_elastic1d)
  ColPass2D colp;                // 2D elastic term: row transforms + one column kernel
  bool use_colpass = false;
  double bn = 0.0, b0 = 0.0;     // its B(k): bn for every k != 0, b0 at k = 0
  double *save_x = nullptr;      // FP32C save steps: FP64 field, dX/dt, mu/M
  std::string kernels;           // text returned by pf5d_stepper_rate_kernels
};

namespace {

constexpr int kTX1 = 128;            // 1D tile
constexpr int kGraphSteps = 50;      // steps per captured graph

// Rate-kernel variants the autotuner chooses from: plane tile (TX x TY
// threads) and the minimum resident blocks per SM (which caps registers);
// fused (one kernel) or split (k_chem64 over all points, then the tile
// kernel reading mu/M back).  All variants compute every value the same way.
struct RateVariant {
  int tx, ty, minb;
  int nth;          // threads of a 2D block (1D block; >= tx * ty)
  bool win;
  bool split;
  bool only3d = false;   // 2D runs another variant's kernels: not tuned there
  bool only2d = false;   // 3D runs another variant's kernels: not tuned there
  size_t smem2d, smem3d;
  void (*set_attrs)(bool vec);
  void (*launch2d)(bool vec, dim3 g, dim3 b, size_t sm, cudaStream_t s, const RateParams &P);
  void (*launch3d)(bool vec, dim3 g, dim3 b, size_t sm, cudaStream_t s, const RateParams &P,
                   int zc);
  std::string (*kernels)(bool vec, int dim);   // the kernel instances of a 2D/3D rate stage
};

// NTH shapes the 2D kernel only (the 3D marching kernel has one thread per
// tile point); SORT applies to both.
template <int TX, int TY, int MINB, bool WIN = true, int NTH = TX * TY, int SORT = 0,
          bool PP = false>
RateVariant make_variant() {
  RateVariant v;
  v.tx = TX;
  v.ty = TY;
  v.minb = MINB;
  v.nth = NTH;
  v.win = WIN;
  v.split = false;
  v.smem2d = tile2d_smem<TX, TY, NTH, SORT>();
  v.smem3d = march3d_smem<TX, TY, SORT>();
  v.set_attrs = [](bool vec) {
    const int s2 = (int)tile2d_smem<TX, TY, NTH, SORT>(), s3 = (int)march3d_smem<TX, TY, SORT>();
    const auto a = cudaFuncAttributeMaxDynamicSharedMemorySize;
    if (vec) {
      cudaFuncSetAttribute(k_rate_tile2d<TX, TY, MINB, true, WIN, false, NTH, SORT, PP>, a, s2);
      cudaFuncSetAttribute(k_rate_march3d<TX, TY, MINB, true, WIN, false, SORT, PP>, a, s3);
    } else {
      cudaFuncSetAttribute(k_rate_tile2d<TX, TY, MINB, false, WIN, false, NTH, SORT, PP>, a, s2);
      cudaFuncSetAttribute(k_rate_march3d<TX, TY, MINB, false, WIN, false, SORT, PP>, a, s3);
    }
  };
  v.launch2d = [](bool vec, dim3 g, dim3 b, size_t sm, cudaStream_t s, const RateParams &P) {
    if (vec) launch_pdl(k_rate_tile2d<TX, TY, MINB, true, WIN, false, NTH, SORT, PP>, g, b, sm, s, P);
    else launch_pdl(k_rate_tile2d<TX, TY, MINB, false, WIN, false, NTH, SORT, PP>, g, b, sm, s, P);
  };
  v.launch3d = [](bool vec, dim3 g, dim3 b, size_t sm, cudaStream_t s, const RateParams &P,
                  int zc) {
    if (vec) launch_pdl(k_rate_march3d<TX, TY, MINB, true, WIN, false, SORT, PP>, g, b, sm, s, P, zc);
    else launch_pdl(k_rate_march3d<TX, TY, MINB, false, WIN, false, SORT, PP>, g, b, sm, s, P, zc);
  };
  v.kernels = [](bool vec, int dim) {
    if (dim == 2) return kname("k_rate_tile2d", {TX, TY, MINB, vec, WIN, 0, NTH, SORT, PP});
    return kname("k_rate_march3d", {TX, TY, MINB, vec, WIN, 0, SORT, PP});
  };
  return v;
}

// The split form's mu/M kernel: k_chem64 (K = 1) or its shared-gather form
// k_chem64i with K points per work item.
template <int DIM, int KMINB, int K = 1>
void launch_chem(bool vec, cudaStream_t s, const RateParams &P) {
  if constexpr (K == 1) {
    const dim3 b(32, 8), g((unsigned)((P.nx + 31) / 32), (unsigned)((P.ny + 7) / 8),
                           (unsigned)P.nz);
    if (vec) launch_pdl(k_chem64<DIM, true, KMINB>, g, b, 0, s, P);
    else launch_pdl(k_chem64<DIM, false, KMINB>, g, b, 0, s, P);
  } else {
    using G = Chem64Geom<DIM, K>;
    const dim3 g((unsigned)((P.nx + G::BX - 1) / G::BX), (unsigned)((P.ny + G::BY - 1) / G::BY),
                 (unsigned)((P.nz + G::BZ - 1) / G::BZ));
    if (vec) launch_pdl(k_chem64i<DIM, true, K, KMINB>, g, dim3(kChem64Threads), G::smem, s, P);
    else launch_pdl(k_chem64i<DIM, false, K, KMINB>, g, dim3(kChem64Threads), G::smem, s, P);
  }
}

template <int DIM, int KMINB, int K>
void chem_attrs() {
  if constexpr (K > 1) {
    const auto a = cudaFuncAttributeMaxDynamicSharedMemorySize;
    cudaFuncSetAttribute(k_chem64i<DIM, true, K, KMINB>, a, (int)Chem64Geom<DIM, K>::smem);
    cudaFuncSetAttribute(k_chem64i<DIM, false, K, KMINB>, a, (int)Chem64Geom<DIM, K>::smem);
  }
}

template <int TX, int TY, int MINB, int KMINB, bool PP = false, int K = 1>
RateVariant make_split_variant() {
  RateVariant v;
  v.tx = TX;
  v.ty = TY;
  v.minb = MINB;
  v.nth = TX * TY;
  v.win = false;
  v.split = true;
  v.smem2d = tile2d_smem<TX, TY>();
  v.smem3d = march3d_smem<TX, TY>();
  v.set_attrs = [](bool) {
    const auto a = cudaFuncAttributeMaxDynamicSharedMemorySize;
    cudaFuncSetAttribute(k_rate_tile2d<TX, TY, MINB, true, false, true>, a,
                         (int)tile2d_smem<TX, TY>());
    cudaFuncSetAttribute(k_rate_march3d<TX, TY, MINB, true, false, true, false, PP>, a,
                         (int)march3d_smem<TX, TY>());
    chem_attrs<2, KMINB, K>();
    chem_attrs<3, KMINB, K>();
  };
  v.launch2d = [](bool vec, dim3 g, dim3 b, size_t sm, cudaStream_t s, const RateParams &P) {
    launch_chem<2, KMINB, K>(vec, s, P);
    launch_pdl(k_rate_tile2d<TX, TY, MINB, true, false, true>, g, b, sm, s, P);
  };
  v.launch3d = [](bool vec, dim3 g, dim3 b, size_t sm, cudaStream_t s, const RateParams &P,
                  int zc) {
    launch_chem<3, KMINB, K>(vec, s, P);
    launch_pdl(k_rate_march3d<TX, TY, MINB, true, false, true, false, PP>, g, b, sm, s, P, zc);
  };
  v.kernels = [](bool vec, int dim) {
    const std::string chem = (K == 1 ? kname("k_chem64", {dim, vec, KMINB})
                                     : kname("k_chem64i", {dim, vec, K, KMINB})) + " + ";
    if (dim == 2) return chem + kname("k_rate_tile2d", {TX, TY, MINB, 1, 0, 1, TX * TY, 0, 0});
    return chem + kname("k_rate_march3d", {TX, TY, MINB, 1, 0, 1, 0, PP});
  };
  return v;
}

// Split variant for 3D with the cp.async marching flux kernel k_flux3_64
// (PP: per-point faces) after the mu/M kernel CHEM (0: k_chem64, 1:
// k_chem64s; k_chem64 for tables that are not double2-aligned); in 2D it
// runs make_split_variant's kernels.
template <int DIM, int KMINB, int CHEM>
void launch_chem3(bool vec, cudaStream_t s, const RateParams &P) {
  if (CHEM == 0 || !vec) {
    launch_chem<DIM, KMINB, 1>(vec, s, P);
    return;
  }
  const dim3 b(32, 8), g((unsigned)((P.nx + 31) / 32), (unsigned)((P.ny + 7) / 8), (unsigned)P.nz);
  launch_pdl(k_chem64s<DIM, KMINB>, g, b, 0, s, P);
}

// Split variant for 2D with k_chem64s (coalesced mu/M rows) before the
// split tile kernel; in 3D it runs make_split_variant's kernels.
template <int TX, int TY, int MINB, int KMINB>
RateVariant make_split2s_variant() {
  RateVariant v = make_split_variant<TX, TY, MINB, KMINB>();
  v.only2d = true;
  v.launch2d = [](bool vec, dim3 g, dim3 b, size_t sm, cudaStream_t s, const RateParams &P) {
    launch_chem3<2, KMINB, 1>(vec, s, P);
    launch_pdl(k_rate_tile2d<TX, TY, MINB, true, false, true>, g, b, sm, s, P);
  };
  v.kernels = [](bool vec, int dim) {
    if (dim == 2)
      return (vec ? kname("k_chem64s", {2, KMINB}) : kname("k_chem64", {2, vec, KMINB})) + " + " +
             kname("k_rate_tile2d", {TX, TY, MINB, 1, 0, 1, TX * TY, 0, 0});
    return kname("k_chem64", {dim, vec, KMINB}) + " + " +
           kname("k_rate_march3d", {TX, TY, MINB, 1, 0, 1, 0, 0});
  };
  return v;
}

template <int TX, int TY, int MINB, int KMINB, bool PP, int CHEM = 0>
RateVariant make_split3_variant() {
  RateVariant v = make_split_variant<TX, TY, MINB, KMINB>();
  v.only3d = true;
  v.smem3d = Flux3Geom64<TX, TY>::smem(PP);
  v.set_attrs = [](bool) {
    const auto a = cudaFuncAttributeMaxDynamicSharedMemorySize;
    cudaFuncSetAttribute(k_rate_tile2d<TX, TY, MINB, true, false, true>, a,
                         (int)tile2d_smem<TX, TY>());
    cudaFuncSetAttribute(k_flux3_64<TX, TY, MINB, PP>, a, (int)Flux3Geom64<TX, TY>::smem(PP));
  };
  v.launch3d = [](bool vec, dim3 g, dim3 b, size_t sm, cudaStream_t s, const RateParams &P,
                  int zc) {
    launch_chem3<3, KMINB, CHEM>(vec, s, P);
    launch_pdl(k_flux3_64<TX, TY, MINB, PP>, g, b, sm, s, P, zc);
  };
  v.kernels = [](bool vec, int dim) {
    const std::string chem =
        (CHEM == 0 || !vec ? kname("k_chem64", {dim, vec, KMINB})
                           : kname("k_chem64s", {dim, KMINB})) + " + ";
    if (dim == 2) return chem + kname("k_rate_tile2d", {TX, TY, MINB, 1, 0, 1, TX * TY, 0, 0});
    return chem + kname("k_flux3_64", {TX, TY, MINB, PP});
  };
  return v;
}

const std::vector<RateVariant> &rate_variants() {
  static const std::vector<RateVariant> v = {
      make_variant<32, 8, 2>(), make_variant<32, 8, 3>(), make_variant<32, 4, 4>(),
      make_variant<16, 8, 4>(), make_variant<64, 4, 2>(), make_variant<32, 4, 6>(),
      make_variant<32, 8, 2, false>(), make_variant<32, 8, 3, false>(),
      make_split_variant<32, 8, 3, 2>(), make_split_variant<32, 8, 3, 3>(),
      make_split_variant<32, 4, 4, 2>(), make_split_variant<32, 4, 4, 3>(),
      make_split_variant<32, 8, 3, 4>(), make_split_variant<32, 4, 4, 4>(),
      make_variant<32, 8, 2, true, 352, true>(), make_variant<32, 8, 2, false, 352, true>(),
      make_variant<32, 8, 2, true, 352, false>(), make_variant<32, 4, 4, true, 224, true>(),
      make_variant<32, 4, 4, false, 224, true>(), make_variant<32, 16, 1, false, 608, true>(),
      make_variant<32, 8, 2, false, 352, true, true>(), make_variant<32, 8, 2, true, 352, false, true>(),
      make_variant<32, 8, 2, false, 256, 2, true>(), make_variant<32, 8, 2, false, 256, 2, false>(),
      make_variant<32, 4, 4, false, 128, 2, true>(),
      make_variant<32, 8, 3, false, 256, false, true>(), make_variant<64, 4, 2, true, 256, false, true>(),
      make_split_variant<32, 8, 3, 3, true>(), make_split_variant<32, 4, 4, 3, true>(),
      make_split_variant<32, 8, 3, 2, false, 2>(), make_split_variant<32, 4, 4, 2, false, 2>(),
      make_split_variant<32, 8, 3, 2, true, 2>(), make_split_variant<32, 4, 4, 2, true, 2>(),
      make_split3_variant<32, 4, 3, 3, true>(), make_split3_variant<32, 4, 3, 3, false>(),
      make_split3_variant<32, 8, 2, 3, true>(), make_split3_variant<32, 8, 2, 3, false>(),
      make_split3_variant<64, 4, 1, 3, true>(), make_split3_variant<32, 4, 2, 3, true>(),
      make_split3_variant<32, 4, 3, 3, true, 1>(), make_split3_variant<32, 4, 3, 4, true, 1>(),
      make_split3_variant<32, 4, 2, 3, true, 1>(),
      make_split2s_variant<32, 8, 3, 4>()};
  return v;
}

// Grid of the rate kernel of `variant` on this solve (and the axis-0 chunk
// of the 3D marching kernel).
dim3 rate_grid_of(const pf5d_stepper *h, int variant, int *zc_out) {
  const RateParams &P = h->rp;
  *zc_out = 1;
  if (h->d.dim == 1) return dim3((unsigned)((P.nx + kTX1 - 1) / kTX1));
  const RateVariant &v = rate_variants()[variant];
  const unsigned gx = (unsigned)((P.nx + v.tx - 1) / v.tx), gy = (unsigned)((P.ny + v.ty - 1) / v.ty);
  if (h->d.dim == 2) return dim3(gx, gy, 1);
  // Chunk of axis-0 planes per block: ~8 resident-block waves, >= 4 planes.
  const int64_t tiles = (int64_t)gx * gy;
  const int64_t target = (int64_t)sm_count() * v.minb * 4;
  int64_t zc = (tiles * P.nz + target - 1) / target;
  zc = std::max<int64_t>(4, std::min<int64_t>(zc, 64));
  zc = std::min<int64_t>(zc, P.nz);
  *zc_out = (int)zc;
  return dim3(gx, gy, (unsigned)((P.nz + zc - 1) / zc));
}

// Block slots needed by the largest rate grid over all variants.
int64_t max_rate_blocks(const pf5d_stepper *h) {
  int64_t m = 1;
  const int nv = h->d.dim == 1 ? 1 : (int)rate_variants().size();
  for (int v = 0; v < nv; ++v) {
    int zc = 1;
    const dim3 g = rate_grid_of(h, v, &zc);
    m = std::max<int64_t>(m, (int64_t)g.x * g.y * g.z);
  }
  return m;
}

pf5d_status configure_rate(pf5d_stepper *h, int variant) {
  const int dim = h->d.dim;
  const RateParams &P = h->rp;
  h->vec = (P.T.stride % 2 == 0) && (((uintptr_t)P.T.grid & 15) == 0);
  if (dim == 1) {
    h->rate_block = dim3(kTX1);
    h->rate_grid = rate_grid_of(h, 0, &h->zc);
    h->rate_smem = 0;
    return PF5D_OK;
  }
  const auto &vars = rate_variants();
  PF5D_REQUIRE(variant >= 0 && variant < (int)vars.size(), PF5D_ERR_ARG, "bad variant %d",
               variant);
  const RateVariant &v = vars[variant];
  h->variant = variant;
  v.set_attrs(h->vec);
  PF5D_LAUNCHED();
  h->rate_block = dim3(v.tx, v.ty);
  if (dim == 2) h->rate_block = dim3(v.nth);
  h->rate_smem = dim == 2 ? v.smem2d : v.smem3d;
  h->rate_grid = rate_grid_of(h, variant, &h->zc);
  return PF5D_OK;
}

pf5d_status launch_rate(pf5d_stepper *h, cudaStream_t s) {
  const dim3 g = h->rate_grid, b = h->rate_block;
  const size_t sm = h->rate_smem;
  switch (h->d.dim) {
    case 1:
      if (h->vec) launch_pdl(k_rate_1d<kTX1, true>, g, b, 0, s, h->rp);
      else launch_pdl(k_rate_1d<kTX1, false>, g, b, 0, s, h->rp);
      break;
    case 2:
      rate_variants()[h->variant].launch2d(h->vec, g, b, sm, s, h->rp);
      break;
    default:
      rate_variants()[h->variant].launch3d(h->vec, g, b, sm, s, h->rp, h->zc);
  }
  PF5D_LAUNCHED();
  PF5D_CUDA(launch_pdl(k_dt_finish, dim3(1), dim3(kDtThreads), 0, s, h->rp,
                       (int)(g.x * g.y * g.z)));
  return PF5D_OK;
}

pf5d_status graph_for(pf5d_stepper *h, int64_t nsteps, cudaGraphExec_t *out);

constexpr int kTuneFinalists = 6;    // variants timed as whole steps
constexpr int kTuneSteps = 10;       // steps per timed graph

// Time every rate-kernel variant's rate stage on this solve (events on `s`,
// a few reps each); then time the fastest few as captured graphs of whole
// steps (what a run executes: the FFT chain, update and launch chaining
// change the order), each from the same saved state, and keep the fastest.
// The field, s and the step state are restored, so tuning leaves the solve
// where it was; any captured graphs are dropped.
pf5d_status autotune_rate(pf5d_stepper *h, cudaStream_t s, float *best_ms) {
  if (h->d.dim == 1) {
    if (best_ms) *best_ms = 0.f;
    return PF5D_OK;
  }
  StepState saved;
  PF5D_CUDA(cudaMemcpyAsync(&saved, h->st, sizeof(saved), cudaMemcpyDeviceToHost, s));
  PF5D_CUDA(cudaStreamSynchronize(s));
  cudaEvent_t e0, e1;
  PF5D_CUDA(cudaEventCreate(&e0));
  PF5D_CUDA(cudaEventCreate(&e1));
  const int reps = 5;
  std::vector<std::pair<float, int>> rate_t;
  for (int v = 0; v < (int)rate_variants().size(); ++v) {
    if (rate_variants()[v].only3d && h->d.dim != 3) continue;
    if (rate_variants()[v].only2d && h->d.dim != 2) continue;
    pf5d_status st = configure_rate(h, v);
    if (st != PF5D_OK) continue;
    if (launch_rate(h, s) != PF5D_OK) {           // warm-up (e.g. too much smem)
      cudaGetLastError();
      continue;
    }
    PF5D_CUDA(cudaEventRecord(e0, s));
    for (int r = 0; r < reps; ++r)
      if ((st = launch_rate(h, s)) != PF5D_OK) break;
    PF5D_CUDA(cudaEventRecord(e1, s));
    PF5D_CUDA(cudaEventSynchronize(e1));
    float ms = 0.f;
    PF5D_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    if (st == PF5D_OK) rate_t.push_back({ms / reps, v});
  }
  PF5D_REQUIRE(!rate_t.empty(), PF5D_ERR_CUDA, "no rate variant ran");
  std::sort(rate_t.begin(), rate_t.end());
  // whole steps of the finalists, each from the saved field / s / state
  const size_t nx = (size_t)h->npts * 4, ns = h->d.elastic ? (size_t)h->npts : 0;
  double *keep = nullptr;
  PF5D_CUDA(cudaMalloc(&keep, (nx + ns) * sizeof(double)));
  auto restore = [&]() {
    cudaMemcpyAsync(h->X, keep, nx * sizeof(double), cudaMemcpyDeviceToDevice, s);
    if (ns) cudaMemcpyAsync(h->s, keep + nx, ns * sizeof(double), cudaMemcpyDeviceToDevice, s);
    cudaMemcpyAsync(h->st, &saved, sizeof(saved), cudaMemcpyHostToDevice, s);
    return cudaGetLastError();
  };
  cudaError_t e = cudaMemcpyAsync(keep, h->X, nx * sizeof(double), cudaMemcpyDeviceToDevice, s);
  if (e == cudaSuccess && ns)
    e = cudaMemcpyAsync(keep + nx, h->s, ns * sizeof(double), cudaMemcpyDeviceToDevice, s);
  int best = rate_t[0].second;
  float best_t = 1e30f;
  const int nfin = std::min<int>((int)rate_t.size(), kTuneFinalists);
  for (int i = 0; i < nfin && e == cudaSuccess; ++i) {
    const int v = rate_t[i].second;
    for (auto &kv : h->graphs) cudaGraphExecDestroy(kv.second);
    h->graphs.clear();
    cudaGraphExec_t g = nullptr;
    if (configure_rate(h, v) != PF5D_OK || graph_for(h, kTuneSteps, &g) != PF5D_OK) continue;
    if ((e = restore()) != cudaSuccess || (e = cudaGraphLaunch(g, s)) != cudaSuccess) break;
    if ((e = restore()) != cudaSuccess || (e = cudaEventRecord(e0, s)) != cudaSuccess ||
        (e = cudaGraphLaunch(g, s)) != cudaSuccess || (e = cudaEventRecord(e1, s)) != cudaSuccess ||
        (e = cudaEventSynchronize(e1)) != cudaSuccess)
      break;
    StepState after;
    float ms = 0.f;
    if ((e = cudaMemcpy(&after, h->st, sizeof(after), cudaMemcpyDeviceToHost)) != cudaSuccess ||
        (e = cudaEventElapsedTime(&ms, e0, e1)) != cudaSuccess)
      break;
    if (!after.halt && ms / kTuneSteps < best_t) {
      best_t = ms / kTuneSteps;
      best = v;
    }
  }
  if (e == cudaSuccess) e = restore();
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  cudaFree(keep);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  PF5D_REQUIRE(e == cudaSuccess, PF5D_ERR_CUDA, "autotune: %s", cudaGetErrorString(e));
  for (auto &kv : h->graphs) cudaGraphExecDestroy(kv.second);
  h->graphs.clear();
  pf5d_status st = configure_rate(h, best);
  if (st != PF5D_OK) return st;
  if (best_ms) *best_ms = best_t;
  return PF5D_OK;
}

// The elastic term of a step: s (the misfit the update wrote) -> s' in
// place, by cuFFT D2Z, the B(k)/N multiply and Z2D, or in 1D by
// k_elastic1d (elastic.py:250-263 with a B(k) that is one constant for
// every k != 0: irfft(B rfft(s)) = bn (s - mean s) + b0 mean s exactly).
pf5d_status elastic_stage(pf5d_stepper *h, cudaStream_t s) {
  if (h->closed1d) {
    PF5D_CUDA(launch_pdl(k_elastic1d, dim3(1), dim3(kElastic1dThreads), 0, s, h->s, h->npts,
                         h->bn, h->b0, (const unsigned *)&h->st->halt));
    return PF5D_OK;
  }
  pf5d_status st;
  if (h->use_colpass) {
    if ((st = colpass_rows_forward(&h->colp, h->s, h->k, s)) != PF5D_OK) return st;
    if ((st = colpass_columns(&h->colp, h->k, h->bk, &h->st->halt, s)) != PF5D_OK) return st;
    return colpass_rows_inverse(&h->colp, h->k, h->s, s);
  }
  if ((st = fft_forward(&h->fft, h->s, h->k, s)) != PF5D_OK) return st;
  if ((st = launch_bmul(h->k, h->bk, h->fft.nk, &h->st->halt, s)) != PF5D_OK) return st;
  return fft_inverse(&h->fft, h->k, h->s, s);
}

pf5d_status enqueue_step(pf5d_stepper *h, cudaStream_t s) {
  pf5d_status st;
  if (h->d.elastic && (st = elastic_stage(h, s)) != PF5D_OK) return st;
  if ((st = launch_rate(h, s)) != PF5D_OK) return st;
  PF5D_CUDA(launch_pdl(k_update_step, dim3(grid_for(h->npts, 256, 4)), dim3(256), 0, s, h->up));
  return PF5D_OK;
}

pf5d_status graph_for(pf5d_stepper *h, int64_t nsteps, cudaGraphExec_t *out) {
  auto it = h->graphs.find(nsteps);
  if (it != h->graphs.end()) {
    *out = it->second;
    return PF5D_OK;
  }
  cudaGraph_t g = nullptr;
  PF5D_CUDA(cudaStreamBeginCapture(h->cap, cudaStreamCaptureModeThreadLocal));
  pf5d_status st = PF5D_OK;
  for (int64_t i = 0; i < nsteps && st == PF5D_OK; ++i) st = enqueue_step(h, h->cap);
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
  h->graphs[nsteps] = exec;
  *out = exec;
  return PF5D_OK;
}

}  // namespace

extern "C" {

pf5d_status pf5d_stepper_create(const pf5d_stepper_desc *desc, double *X, void *stream,
                                pf5d_stepper **out) {
  PF5D_REQUIRE(desc && X && out, PF5D_ERR_ARG, "null argument");
  PF5D_REQUIRE(desc->dim >= 1 && desc->dim <= 3, PF5D_ERR_DIM,
               "Unsupported system_dim=%d. Choose 1, 2, or 3.", desc->dim);
  PF5D_REQUIRE(desc->precision == PF5D_PRECISION_FP64 || desc->precision == PF5D_PRECISION_FP32C,
               PF5D_ERR_ARG, "unknown precision %d", desc->precision);
  for (int d = 0; d < desc->dim; ++d)
    PF5D_REQUIRE(desc->shape[d] > 0 && desc->shape[d] <= (1LL << 30), PF5D_ERR_ARG, "bad shape");
  PF5D_REQUIRE(!desc->elastic || desc->bk, PF5D_ERR_ARG, "elastic term needs B(k)");
  if (desc->precision == PF5D_PRECISION_FP32C) {
    PF5D_REQUIRE(desc->node_coord && desc->table_n >= 2, PF5D_ERR_ARG, "bad table description");
    auto *h = new pf5d_stepper();
    h->d = *desc;
    h->d.bk = nullptr;
    h->X = X;
    pf5d_status st = s32_create(desc, X, stream, &h->s32);
    if (st != PF5D_OK) {
      delete h;
      return st;
    }
    *out = h;
    return PF5D_OK;
  }
  PF5D_REQUIRE(desc->grid && desc->node_coord && desc->nprops == NP &&
                   desc->node_stride >= NP && desc->table_n >= 2,
               PF5D_ERR_ARG, "bad table description");
  PF5D_REQUIRE(!desc->elastic || desc->bk, PF5D_ERR_ARG, "elastic term needs B(k)");
  PF5D_REQUIRE(((uintptr_t)X & 15) == 0, PF5D_ERR_ARG, "X must be 16-byte aligned");
  auto *h = new pf5d_stepper();
  h->d = *desc;
  h->d.bk = nullptr;
  h->X = X;
  int64_t npts = 1;
  for (int d = 0; d < desc->dim; ++d) {
    if (desc->shape[d] <= 0 || desc->shape[d] > (1LL << 30)) {
      delete h;
      set_error("bad shape");
      return PF5D_ERR_ARG;
    }
    h->shape[d] = desc->shape[d];
    npts *= desc->shape[d];
  }
  h->npts = npts;
  cudaStream_t s = as_stream(stream);
  pf5d_status st = PF5D_OK;
  auto fail = [&](pf5d_status code) {
    pf5d_stepper_destroy(h);
    return code;
  };
  if (cudaMalloc(&h->dX, npts * 4 * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&h->st, sizeof(StepState)) != cudaSuccess ||
      cudaStreamCreateWithFlags(&h->cap, cudaStreamNonBlocking) != cudaSuccess) {
    set_error("device allocation failed");
    return fail(PF5D_ERR_CUDA);
  }
  if (cudaMalloc(&h->mm, (size_t)npts * NP * sizeof(double)) != cudaSuccess) {
    set_error("device allocation failed");
    return fail(PF5D_ERR_CUDA);
  }
  if (desc->elastic && desc->dim == 1 && npts <= kElastic1dMax) {
    // B(k) of a 1D solve depends on k only through its sign: one value for
    // every k != 0 (checked exactly here), so the closed form applies
    const int64_t nk = npts / 2 + 1;
    bool flat = true;
    for (int64_t i = 2; i < nk && flat; ++i) flat = desc->bk[i] == desc->bk[1];
    h->closed1d = flat;
    h->bn = nk > 1 ? desc->bk[1] : 0.0;
    h->b0 = desc->bk[0];
  }
  if (desc->elastic) {
    if ((st = fft_create(desc->dim, h->shape, &h->fft)) != PF5D_OK) return fail(st);
    if ((st = upload_bk_scaled(desc->bk, h->fft.nk, npts, &h->bk)) != PF5D_OK) return fail(st);
    const int64_t n0 = h->shape[0];
    if (desc->dim == 2 && n0 >= 8 && n0 <= 1024 && (n0 & (n0 - 1)) == 0) {
      h->use_colpass = colpass_create(h->shape, &h->colp, false) == PF5D_OK;
      if (!h->use_colpass) colpass_destroy(&h->colp);
    }
    if (cudaMalloc(&h->s, npts * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&h->k, h->fft.nk * sizeof(cufftDoubleComplex)) != cudaSuccess) {
      set_error("device allocation failed");
      return fail(PF5D_ERR_CUDA);
    }
  }
  RateParams &P = h->rp;
  if (desc->dim == 1) {
    P.nz = 1; P.ny = 1; P.nx = (int)h->shape[0];
  } else if (desc->dim == 2) {
    P.nz = 1; P.ny = (int)h->shape[0]; P.nx = (int)h->shape[1];
  } else {
    P.nz = (int)h->shape[0]; P.ny = (int)h->shape[1]; P.nx = (int)h->shape[2];
  }
  P.X = X;
  P.sp = desc->elastic ? h->s : nullptr;
  P.dX = h->dX;
  P.T.grid = desc->grid;
  P.T.coord = desc->node_coord;
  P.T.n = desc->table_n;
  P.T.stride = desc->node_stride;
  P.T.inv_step = 1.0 / desc->resolution;
  P.T.threshold = 1.0 - 4.0 * desc->resolution - 1e-9;
  P.T.max_nn_dist = desc->max_nn_dist;
  for (int c = 0; c < 4; ++c) {
    P.kappa.v[c] = desc->kappa[c];
    P.lvec.v[c] = desc->lvec[c];
  }
  P.inv_dx = 1.0 / desc->dx;
  P.inv_dx2 = 1.0 / (desc->dx * desc->dx);
  P.ctld = desc->ctld;
  P.t_cfl = desc->t_cfl;
  P.lower = desc->lower_limit;
  P.upper = desc->upper_limit;
  P.factor = desc->max_change_factor;
  P.adaptive = desc->adaptive;
  P.st = h->st;
  P.mm = h->mm;
  P.npts = npts;
  if (cudaMalloc(&h->partial, (size_t)max_rate_blocks(h) * sizeof(double)) != cudaSuccess) {
    set_error("device allocation failed");
    return fail(PF5D_ERR_CUDA);
  }
  P.partial = h->partial;
  UpdateParams &U = h->up;
  U.X = X;
  U.dX = h->dX;
  U.npts = npts;
  U.st = h->st;
  for (int c = 0; c < 4; ++c) {
    U.x0.v[c] = desc->x0[c];
    U.lvec.v[c] = desc->lvec[c];
  }
  U.s = desc->elastic ? h->s : nullptr;
  U.oob_interval = desc->oob_interval;
  if ((st = configure_rate(h, 0)) != PF5D_OK) return fail(st);
  if ((st = pf5d_stepper_reset(h, desc->dt0, 0.0, stream)) != PF5D_OK) return fail(st);
  (void)s;
  *out = h;
  return PF5D_OK;
}

pf5d_status pf5d_stepper_reset(pf5d_stepper *h, double dt, double time, void *stream) {
  PF5D_REQUIRE(h, PF5D_ERR_ARG, "null stepper");
  if (h->s32) return s32_reset(h->s32, h->X, dt, time, stream);
  cudaStream_t s = as_stream(stream);
  StepState init{};
  init.dt = dt;
  init.time = time;
  PF5D_CUDA(cudaMemcpyAsync(h->st, &init, sizeof(init), cudaMemcpyHostToDevice, s));
  if (h->d.oob_interval > 0) {
    k_check_state<<<grid_for(h->npts, 256, 2), 256, 0, s>>>(h->X, h->npts, h->st);
    PF5D_LAUNCHED();
  }
  if (h->d.elastic) {
    Vec4 x0, l;
    for (int c = 0; c < 4; ++c) {
      x0.v[c] = h->d.x0[c];
      l.v[c] = h->d.lvec[c];
    }
    pf5d_status st = launch_misfit(h->X, h->npts, x0, l, h->s, nullptr, s);
    if (st != PF5D_OK) return st;
  }
  PF5D_CUDA(cudaStreamSynchronize(s));
  return PF5D_OK;
}

pf5d_status pf5d_stepper_advance(pf5d_stepper *h, int64_t nsteps, void *stream) {
  PF5D_REQUIRE(h && nsteps >= 0, PF5D_ERR_ARG, "bad arguments");
  if (h->s32) return s32_advance(h->s32, nsteps, stream);
  cudaStream_t s = as_stream(stream);
  while (nsteps > 0) {
    const int64_t n = nsteps < kGraphSteps ? nsteps : kGraphSteps;
    cudaGraphExec_t g = nullptr;
    pf5d_status st = graph_for(h, n, &g);
    if (st != PF5D_OK) return st;
    PF5D_CUDA(cudaGraphLaunch(g, s));
    nsteps -= n;
  }
  return PF5D_OK;
}

pf5d_status pf5d_stepper_state(pf5d_stepper *h, pf5d_step_state *out, void *stream) {
  PF5D_REQUIRE(h && out, PF5D_ERR_ARG, "bad arguments");
  if (h->s32) return s32_state(h->s32, out, stream);
  StepState hs;
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

double *pf5d_stepper_rate(pf5d_stepper *h) {
  if (!h) return nullptr;
  if (h->s32) return reinterpret_cast<double *>(s32_rate(h->s32));
  return h->dX;
}

pf5d_status pf5d_stepper_field(pf5d_stepper *h, double *X_out, void *stream) {
  PF5D_REQUIRE(h && X_out, PF5D_ERR_ARG, "bad arguments");
  if (h->s32) return s32_field(h->s32, X_out, stream);
  if (X_out != h->X)
    PF5D_CUDA(cudaMemcpyAsync(X_out, h->X, h->npts * 4 * sizeof(double), cudaMemcpyDeviceToDevice,
                              as_stream(stream)));
  return PF5D_OK;
}

pf5d_status pf5d_stepper_mass(pf5d_stepper *h, double *mean_out, void *stream) {
  PF5D_REQUIRE(h && mean_out, PF5D_ERR_ARG, "bad arguments");
  if (h->s32) return s32_mass(h->s32, mean_out, stream);
  cudaStream_t s = as_stream(stream);
  if (!h->mass_ws) PF5D_CUDA(cudaMalloc(&h->mass_ws, (kMeanBlocks * S + S) * sizeof(double)));
  const unsigned nb = std::min<unsigned>(kMeanBlocks, grid_for(h->npts, 256, 4));
  k_mean_partial<<<nb, 256, 0, s>>>(h->X, h->npts, h->mass_ws);
  PF5D_LAUNCHED();
  k_mean_final<<<1, 32, 0, s>>>(h->mass_ws, (int)nb, h->mass_ws + kMeanBlocks * S);
  PF5D_LAUNCHED();
  double sums[S];
  PF5D_CUDA(cudaMemcpyAsync(sums, h->mass_ws + kMeanBlocks * S, sizeof(sums),
                            cudaMemcpyDeviceToHost, s));
  PF5D_CUDA(cudaStreamSynchronize(s));
  for (int c = 0; c < S; ++c) mean_out[c] = sums[c] / (double)h->npts;
  return PF5D_OK;
}

pf5d_status pf5d_stepper_autotune(pf5d_stepper *h, int32_t *variant, float *best_ms,
                                  void *stream) {
  PF5D_REQUIRE(h, PF5D_ERR_ARG, "null stepper");
  if (h->s32) return s32_autotune(h->s32, variant, best_ms, stream);
  pf5d_status st = autotune_rate(h, as_stream(stream), best_ms);
  if (variant) *variant = h->variant;
  return st;
}

pf5d_status pf5d_stepper_set_variant(pf5d_stepper *h, int32_t variant) {
  PF5D_REQUIRE(h, PF5D_ERR_ARG, "null stepper");
  if (h->s32) return s32_set_variant(h->s32, variant);
  pf5d_status st = configure_rate(h, variant);
  if (st != PF5D_OK) return st;
  for (auto &kv : h->graphs) cudaGraphExecDestroy(kv.second);
  h->graphs.clear();
  return PF5D_OK;
}

pf5d_status pf5d_stepper_step_save(pf5d_stepper *h, pf5d_save_diag *out, void *stream) {
  PF5D_REQUIRE(h && out, PF5D_ERR_ARG, "bad arguments");
  cudaStream_t s = as_stream(stream);
  std::memset(out, 0, sizeof(*out));
  pf5d_step_state before, after;
  pf5d_status st = pf5d_stepper_state(h, &before, stream);
  if (st != PF5D_OK) return st;
  out->step = before.step;
  if (before.halted) {
    out->halted = 1;
    out->dt = before.dt;
    out->time = before.time;
    return PF5D_OK;
  }
  DiagGeom G;
  const int dim = h->d.dim;
  G.nz = dim == 3 ? (int)h->d.shape[0] : 1;
  G.ny = dim == 1 ? 1 : (int)h->d.shape[dim - 2];
  G.nx = (int)h->d.shape[dim - 1];
  G.dim = dim;
  G.npts = (int64_t)G.nz * G.ny * G.nx;
  G.inv_dx = 1.0 / h->d.dx;
  G.inv_dx2 = 1.0 / (h->d.dx * h->d.dx);
  for (int c = 0; c < S; ++c) G.kappa[c] = h->d.kappa[c];
  const int rows = kDiagBlocks;
  if (!h->diag_ws)
    PF5D_CUDA(cudaMalloc(&h->diag_ws, (size_t)(rows * (kDiagPre + kDiagPost + kDiagVar) + S) *
                                          sizeof(double)));
  double *pre = h->diag_ws, *post = pre + rows * kDiagPre, *var = post + rows * kDiagPost;
  double *mean = var + rows * kDiagVar;
  const unsigned nb = std::min<unsigned>(rows, grid_for(G.npts, kDiagThreads, 1));
  const double *Xpre, *dXpre, *mmpre, *Xpost;
  if (h->s32) {
    // FP32-compensated form: FP64 copies of the field, dX/dt and mu/M
    if (!h->save_x) {
      PF5D_CUDA(cudaMalloc(&h->save_x, (size_t)G.npts * (4 + 4 + NP) * sizeof(double)));
    }
    double *sx = h->save_x, *sdx = sx + 4 * G.npts, *smm = sdx + 4 * G.npts;
    if ((st = s32_step_save_inputs(h->s32, sx, sdx, smm, stream)) != PF5D_OK) return st;
    k_diag_pre<<<nb, kDiagThreads, 0, s>>>(G, sx, sdx, smm, pre);
    PF5D_LAUNCHED();
    if ((st = s32_step_update(h->s32, stream)) != PF5D_OK) return st;
    if ((st = s32_field(h->s32, sx, stream)) != PF5D_OK) return st;
    Xpost = sx;
  } else {
    // the step up to its rate evaluation, as enqueue_step
    if (h->d.elastic && (st = elastic_stage(h, s)) != PF5D_OK) return st;
    if ((st = launch_rate(h, s)) != PF5D_OK) return st;
    // mu and M of this step at every point, then the "before" reductions
    switch (dim) {
      case 1: launch_chem<1, 3>(h->vec, s, h->rp); break;
      case 2: launch_chem<2, 3>(h->vec, s, h->rp); break;
      default: launch_chem<3, 3>(h->vec, s, h->rp);
    }
    PF5D_LAUNCHED();
    Xpre = h->X;
    dXpre = h->dX;
    mmpre = h->mm;
    k_diag_pre<<<nb, kDiagThreads, 0, s>>>(G, Xpre, dXpre, mmpre, pre);
    PF5D_LAUNCHED();
    k_update_step<<<grid_for(h->npts, 256, 4), 256, 0, s>>>(h->up);
    PF5D_LAUNCHED();
    Xpost = h->X;
  }
  k_diag_post<<<nb, kDiagThreads, 0, s>>>(G, Xpost, post);
  PF5D_LAUNCHED();
  std::vector<double> hp((size_t)nb * kDiagPre), hq((size_t)nb * kDiagPost);
  PF5D_CUDA(cudaMemcpyAsync(hp.data(), pre, hp.size() * sizeof(double), cudaMemcpyDeviceToHost, s));
  PF5D_CUDA(cudaMemcpyAsync(hq.data(), post, hq.size() * sizeof(double), cudaMemcpyDeviceToHost, s));
  PF5D_CUDA(cudaStreamSynchronize(s));
  if ((st = pf5d_stepper_state(h, &after, stream)) != PF5D_OK) return st;
  for (int c = 0; c < S; ++c) {
    double net = 0.0, mx = 0.0, tf = 0.0, mass = 0.0, nmn = -INFINITY, mxx = -INFINITY;
    for (unsigned b = 0; b < nb; ++b) {
      net += hp[b * kDiagPre + c];
      mx = std::max(mx, hp[b * kDiagPre + S + c]);
      tf += hp[b * kDiagPre + 2 * S + c];
      mass += hq[b * kDiagPost + c];
      nmn = std::max(nmn, hq[b * kDiagPost + S + c]);
      mxx = std::max(mxx, hq[b * kDiagPost + 2 * S + c]);
    }
    out->net[c] = net;
    out->max_change[c] = mx;
    out->total_flux[c] = tf;
    out->mass[c] = mass;
    out->comp_min[c] = -nmn;
    out->comp_max[c] = mxx;
  }
  double msum = -INFINITY, fg = 0.0;
  for (unsigned b = 0; b < nb; ++b) {
    msum = std::max(msum, hq[b * kDiagPost + 3 * S]);
    fg += hq[b * kDiagPost + 3 * S + 1];
  }
  out->comp_fe_min = 1.0 - msum;
  double cell = 1.0;
  for (int d = 0; d < dim; ++d) cell *= h->d.dx;
  out->f_grad = -0.5 * cell * fg;
  double m[S];
  for (int c = 0; c < S; ++c) m[c] = out->mass[c] / (double)G.npts;
  PF5D_CUDA(cudaMemcpyAsync(mean, m, sizeof(m), cudaMemcpyHostToDevice, s));
  k_diag_var<<<nb, kDiagThreads, 0, s>>>(G, Xpost, mean, var);
  PF5D_LAUNCHED();
  std::vector<double> hv((size_t)nb * kDiagVar);
  PF5D_CUDA(cudaMemcpyAsync(hv.data(), var, hv.size() * sizeof(double), cudaMemcpyDeviceToHost, s));
  PF5D_CUDA(cudaStreamSynchronize(s));
  for (int c = 0; c < S; ++c) {
    double v = 0.0;
    for (unsigned b = 0; b < nb; ++b) v += hv[b * kDiagVar + c];
    out->comp_var[c] = v / (double)G.npts;
  }
  out->xdotmax = after.xdotmax;
  out->dt = after.dt;
  out->time = after.time;
  out->halted = 0;          // the step ran; a halt it raised shows in the next state
  return PF5D_OK;
}

int32_t pf5d_stepper_launches_per_step(const pf5d_stepper *h) {
  if (!h) return 0;
  if (h->s32) return s32_launches_per_step(h->s32);
  const bool split = h->d.dim >= 2 && rate_variants()[h->variant].split;
  return (split ? 2 : 1) + 2 + (h->d.elastic ? 1 : 0);   // rate (+chem), dt, update, bmul
}

const char *pf5d_stepper_rate_kernels(pf5d_stepper *h) {
  if (!h) return "";
  if (h->s32) return s32_rate_kernels(h->s32);
  if (h->d.dim == 1) h->kernels = kname("k_rate_1d", {kTX1, h->vec});
  else h->kernels = rate_variants()[h->variant].kernels(h->vec, h->d.dim);
  h->kernels += " + k_dt_finish";
  return h->kernels.c_str();
}

int32_t pf5d_stepper_variant_count(const pf5d_stepper *h) {
  if (!h) return 0;
  return h->s32 ? s32_variant_count() : (int32_t)rate_variants().size();
}

pf5d_status pf5d_stepper_launch_stage(pf5d_stepper *h, int32_t stage, void *stream) {
  PF5D_REQUIRE(h, PF5D_ERR_ARG, "null stepper");
  if (h->s32) return s32_launch_stage(h->s32, stage, stream);
  cudaStream_t s = as_stream(stream);
  switch (stage) {
    case PF5D_STAGE_RATE:
      return launch_rate(h, s);
    case PF5D_STAGE_UPDATE:
      k_update_step<<<grid_for(h->npts, 256, 4), 256, 0, s>>>(h->up);
      PF5D_LAUNCHED();
      return PF5D_OK;
    // 1D closed form: the whole elastic term is the FFT_FWD stage
    case PF5D_STAGE_FFT_FWD:
      PF5D_REQUIRE(h->d.elastic, PF5D_ERR_ARG, "elasticity is off");
      if (h->closed1d) return elastic_stage(h, s);
      if (h->use_colpass) return colpass_rows_forward(&h->colp, h->s, h->k, s);
      return fft_forward(&h->fft, h->s, h->k, s);
    case PF5D_STAGE_BMUL:
      PF5D_REQUIRE(h->d.elastic, PF5D_ERR_ARG, "elasticity is off");
      if (h->closed1d) return PF5D_OK;
      if (h->use_colpass) return colpass_columns(&h->colp, h->k, h->bk, &h->st->halt, s);
      return launch_bmul(h->k, h->bk, h->fft.nk, &h->st->halt, s);
    case PF5D_STAGE_FFT_INV:
      PF5D_REQUIRE(h->d.elastic, PF5D_ERR_ARG, "elasticity is off");
      if (h->closed1d) return PF5D_OK;
      if (h->use_colpass) return colpass_rows_inverse(&h->colp, h->k, h->s, s);
      return fft_inverse(&h->fft, h->k, h->s, s);
    default:
      set_error("unknown stage %d", stage);
      return PF5D_ERR_ARG;
  }
}

pf5d_status pf5d_stepper_destroy(pf5d_stepper *h) {
  if (!h) return PF5D_OK;
  if (h->s32) s32_destroy(h->s32);
  cudaFree(h->mass_ws);
  cudaFree(h->mm);
  cudaFree(h->diag_ws);
  cudaFree(h->partial);
  cudaFree(h->save_x);
  for (auto &kv : h->graphs) cudaGraphExecDestroy(kv.second);
  fft_destroy(&h->fft);
  cudaFree(h->dX);
  cudaFree(h->s);
  cudaFree(h->k);
  cudaFree(h->bk);
  colpass_destroy(&h->colp);
  cudaFree(h->st);
  if (h->cap) cudaStreamDestroy(h->cap);
  delete h;
  return PF5D_OK;
}

}  // extern "C"
