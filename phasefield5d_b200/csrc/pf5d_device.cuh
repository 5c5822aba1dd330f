// pf5d_device.cuh -- FP64 device building blocks shared by every kernel.
//
// Bit-faithfulness: each routine evaluates the reference's expressions in the
// reference's order, one IEEE rounding per operation.  Translation units that
// include this header are compiled with -fmad=false so nvcc never contracts a
// multiply and an add into an FMA (the reference's Numba kernels run with
// fastmath=False, which never contracts either).  Division and square root
// use the IEEE-rounded defaults (-prec-div=true, -prec-sqrt=true).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/pf5d.h"

namespace pf5d {

constexpr int S = 4;    // independent components
constexpr int NM = 5;   // mobilities (Fe first)
constexpr int NP = 9;   // table props: mu1..mu4, M_Fe, M1..M4

// Periodic neighbour indices (phasefield5d/solver/operators.py:45-46 pattern).
__device__ __forceinline__ int64_t wrap_p(int64_t i, int64_t n) { return i + 1 < n ? i + 1 : 0; }
__device__ __forceinline__ int64_t wrap_m(int64_t i, int64_t n) { return i - 1 >= 0 ? i - 1 : n - 1; }
// General periodic index for halo loads (any offset, any n >= 1).
__device__ __forceinline__ int wrap_any(int i, int n) {
  int r = i % n;
  return r < 0 ? r + n : r;
}

// Table view passed by value to kernels.
struct Table {
  const double *grid;       // dense (n,n,n,n,stride)
  const double *coord;      // (n,) stored node coordinate per index
  int n;                    // nodes per axis
  int stride;               // doubles per node
  double inv_step;          // 1.0 / resolution
  double threshold;         // 1.0 - 4.0*resolution - 1e-9
  double max_nn_dist;       // <= 0: unchecked
};

// interpolation.py:110-121
__device__ __forceinline__ void axis_coord(double u, int num, int &i, double &t) {
  if (u <= 0.0) {
    i = 0;
    t = 0.0;
  } else if (u >= (double)(num - 1)) {
    i = num - 2;
    t = 1.0;
  } else {
    i = (int)u;
    t = u - (double)i;
  }
}

// sum_d x[d] from 0.0, left to right (interpolation.py:74-79).
__device__ __forceinline__ bool linear_region(const Table &T, const double x[S]) {
  double s = 0.0;
  s = s + x[0];
  s = s + x[1];
  s = s + x[2];
  s = s + x[3];
  return s <= T.threshold;
}

// Quadrilinear interpolation of NP props at x (interpolation.py:103-147).
// Corner order c = b0 b1 b2 b3 (binary), weights ((w0*w1)*w2)*w3, per-prop
// sum of the 16 terms left to right.  Corners are visited outermost so each
// corner's NP props are one contiguous run of the node.  VEC: the node
// stride is even and the table 16-byte aligned, so a node is read as
// double2 pairs.
template <bool VEC>
__device__ __forceinline__ void interp_linear(const Table &T, const double x[S], double out[NP]) {
  int i0, i1, i2, i3;
  double t0, t1, t2, t3;
  axis_coord(x[0] * T.inv_step, T.n, i0, t0);
  axis_coord(x[1] * T.inv_step, T.n, i1, t1);
  axis_coord(x[2] * T.inv_step, T.n, i2, t2);
  axis_coord(x[3] * T.inv_step, T.n, i3, t3);
  const double q0 = 1.0 - t0, q1 = 1.0 - t1, q2 = 1.0 - t2, q3 = 1.0 - t3;
  const int64_t s3 = T.stride, s2 = (int64_t)T.n * s3, s1 = (int64_t)T.n * s2,
                s0 = (int64_t)T.n * s1;
  const double *base = T.grid + i0 * s0 + i1 * s1 + i2 * s2 + i3 * s3;
#pragma unroll
  for (int c = 0; c < 16; ++c) {
    const int b0 = (c >> 3) & 1, b1 = (c >> 2) & 1, b2 = (c >> 1) & 1, b3 = c & 1;
    const double w = (b0 ? t0 : q0) * (b1 ? t1 : q1) * (b2 ? t2 : q2) * (b3 ? t3 : q3);
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
    for (int p = 0; p < NP; ++p) {
      const double term = w * v[p];
      out[p] = (c == 0) ? term : out[p] + term;
    }
  }
}

// Nearest table row for a point outside the linear region
// (interpolation.py:203-209, cKDTree over the row compositions); returns the
// node index (the caller reads the row).
//
// Rows sit on grid nodes, so the nearest row is the nearest present node
// (the table's first prop is NaN at absent nodes).  The search is exact for
// any finite point, on or far off the simplex:
//   * it scans the window [f_d - r, f_d + r] (clipped to [0, N]) around the
//     point's clamped cell f_d = clamp(floor(x_d / res), 0, N), r = 2 first;
//   * every node outside the window lies farther than `gap`, the distance
//     from x to the nearest excluded coordinate on any axis, so a best
//     squared distance below gap^2 is the global minimum (the comparison is
//     made on the same rounded squares the scan computes, so rounding cannot
//     break it);
//   * otherwise the window grows (r = 8, 32, ...) until the bound holds or
//     the window spans the whole table.
// Per axis the scan walks coordinates upward and stops once a coordinate
// above x already makes the partial distance exceed the best.  Distances
// are sum_d (x_d - c_d)^2 in axis order; of exactly equal distances the
// first node in lexicographic order wins.  A non-finite component returns
// no node with PF5D_FLAG_NN_NONFINITE (cKDTree.query raises ValueError for
// it); a table with no present node returns none with NN_TRUNCATED.
struct NearestNode {
  int64_t node;        // -1: no node (non-finite point or empty table)
  unsigned flags;      // PF5D_FLAG_NN_*
};

// Flags of the fallback that end a step loop where the reference's loop
// raises: a non-finite composition (ValueError from cKDTree.query), a row
// farther than max_nn_dist (RuntimeError, interpolation.py:207-208), and a
// table without rows.
constexpr unsigned kNNErrorFlags = PF5D_FLAG_NN_FAR | PF5D_FLAG_NN_TRUNCATED | PF5D_FLAG_NN_NONFINITE;

// Record a rate kernel's flags in its step state (flags, halt); the
// fallback's error flags halt the loop before the step's update.
template <typename St>
__device__ __forceinline__ void raise_rate_flags(St *st, unsigned f) {
  if (!f) return;
  atomicOr(&st->flags, f);
  if (f & kNNErrorFlags) atomicExch(&st->halt, 1u);
}

// The search needs only the node coordinates and a presence probe, so it
// serves FP64 and FP32 tables alike: `grid` points at the first prop of
// node 0, `stride` is in elements of type E.
template <typename E>
static __device__ __noinline__ NearestNode nearest_node_g(const E *grid, int stride,
                                                          const double *coord, int n_axis,
                                                          double inv_step, double max_nn_dist,
                                                          double x0, double x1, double x2,
                                                          double x3) {
  const double x[S] = {x0, x1, x2, x3};
  NearestNode r{-1, PF5D_FLAG_NN_USED};
  if (!(isfinite(x0) && isfinite(x1) && isfinite(x2) && isfinite(x3))) {
    r.flags |= PF5D_FLAG_NN_NONFINITE;
    return r;
  }
  const int N = n_axis - 1;
  const int64_t n = n_axis;
  int f[S];
#pragma unroll
  for (int d = 0; d < S; ++d) {
    const double u = fmin(fmax(x[d] * inv_step, 0.0), (double)N);
    f[d] = (int)floor(u);
  }
  double best = __longlong_as_double(0x7ff0000000000000LL);   // +inf
  int64_t best_node = -1;
  for (int rad = 2;; rad *= 4) {
    int lo[S], hi[S];
    double gap = __longlong_as_double(0x7ff0000000000000LL);
    bool whole = true;
#pragma unroll
    for (int d = 0; d < S; ++d) {
      lo[d] = max(0, f[d] - rad);
      hi[d] = min(N, f[d] + rad);
      if (lo[d] > 0) {
        gap = fmin(gap, fmax(x[d] - coord[lo[d] - 1], 0.0));
        whole = false;
      }
      if (hi[d] < N) {
        gap = fmin(gap, fmax(coord[hi[d] + 1] - x[d], 0.0));
        whole = false;
      }
    }
    for (int k0 = lo[0]; k0 <= hi[0]; ++k0) {
      const double d0 = x[0] - coord[k0];
      const double e0 = d0 * d0;
      if (e0 > best) {
        if (d0 < 0.0) break;          // coordinates only move away from here on
        continue;
      }
      for (int k1 = lo[1]; k1 <= hi[1]; ++k1) {
        const double d1 = x[1] - coord[k1];
        const double e1 = e0 + d1 * d1;
        if (e1 > best) {
          if (d1 < 0.0) break;
          continue;
        }
        for (int k2 = lo[2]; k2 <= hi[2]; ++k2) {
          const double d2 = x[2] - coord[k2];
          const double e2 = e1 + d2 * d2;
          if (e2 > best) {
            if (d2 < 0.0) break;
            continue;
          }
          for (int k3 = lo[3]; k3 <= hi[3]; ++k3) {
            const double d3 = x[3] - coord[k3];
            const double e3 = e2 + d3 * d3;
            if (e3 > best) {
              if (d3 < 0.0) break;
              continue;
            }
            const int64_t node = ((k0 * n + k1) * n + k2) * n + k3;
            if (e3 < best || node < best_node) {
              const E probe = __ldg(grid + node * stride);
              if (probe == probe) {          // present (not NaN)
                best = e3;
                best_node = node;
              }
            }
          }
        }
      }
    }
    if (whole || (best_node >= 0 && best < gap * gap)) break;
  }
  r.node = best_node;
  if (best_node < 0) r.flags |= PF5D_FLAG_NN_TRUNCATED;
  else if (max_nn_dist > 0.0 && sqrt(best) > max_nn_dist) r.flags |= PF5D_FLAG_NN_FAR;
  return r;
}

__device__ __forceinline__ NearestNode nearest_node(const Table &T, double x0, double x1,
                                                    double x2, double x3) {
  return nearest_node_g<double>(T.grid, T.stride, T.coord, T.n, T.inv_step, T.max_nn_dist, x0,
                                x1, x2, x3);
}

// Interpolation with fallback for one point; returns true on the linear branch.
template <bool VEC = false>
__device__ __forceinline__ bool interp_point(const Table &T, const double x[S], double out[NP],
                                             unsigned *flag_bits) {
  if (linear_region(T, x)) {
    interp_linear<VEC>(T, x, out);
    return true;
  }
  const NearestNode r = nearest_node(T, x[0], x[1], x[2], x[3]);
  *flag_bits |= r.flags;
  const double *row = T.grid + (r.node < 0 ? 0 : r.node) * T.stride;
#pragma unroll
  for (int p = 0; p < NP; ++p)
    out[p] = r.node < 0 ? __longlong_as_double(0x7ff8000000000000LL) : __ldg(row + p);
  return false;
}

// _face_flux (phasefield5d/solver/fluxes.py:128-160) for the face between a
// "centre" point c and a neighbour n, with g = the mu gradient across it.
// J_a = w_fe*(-Xm_a)*(-<Xm,g>) + Xm_a*Mm_{1+a}*(g_a - <Xm,g>) - Xm_a*sum_k(...)
__device__ __forceinline__ void face_flux(const double Xc[S], const double Mc[NM],
                                          const double Xn[S], const double Mn[NM],
                                          const double g[S], double J[S]) {
  double xm[S], mm[NM], dk[S];
#pragma unroll
  for (int a = 0; a < S; ++a) xm[a] = 0.5 * (Xc[a] + Xn[a]);
#pragma unroll
  for (int a = 0; a < NM; ++a) mm[a] = 0.5 * (Mc[a] + Mn[a]);
  double sum_x = 0.0;
#pragma unroll
  for (int a = 0; a < S; ++a) sum_x = sum_x + xm[a];
  const double w_fe = (1.0 - sum_x) * mm[0];
  double dot_xg = 0.0;
#pragma unroll
  for (int b = 0; b < S; ++b) dot_xg = dot_xg + xm[b] * g[b];
  const double dot_fe = -dot_xg;
#pragma unroll
  for (int k = 0; k < S; ++k) dk[k] = g[k] - dot_xg;
  double sum_wk = 0.0;
#pragma unroll
  for (int k = 0; k < S; ++k) sum_wk = sum_wk + xm[k] * mm[1 + k] * dk[k];
#pragma unroll
  for (int a = 0; a < S; ++a) {
    const double wa = xm[a] * mm[1 + a];
    J[a] = w_fe * (-xm[a]) * dot_fe + wa * dk[a] - xm[a] * sum_wk;
  }
}

// apply_adaptive_time (phasefield5d/solver/system.py:90-112); Python's min()
// keeps its first argument unless a later one is strictly smaller, and
// np.clip is minimum(maximum(a, lo), hi).
__host__ __device__ inline double adaptive_dt(double dt, double xdotmax, double ctld, double t_cfl,
                                              double lower, double upper, double factor) {
  double dt_raw;
  if (xdotmax <= 0.0) {
    dt_raw = dt;
  } else {
    double lo = lower / xdotmax, hi = upper / xdotmax;
    if (lo > hi) {
      const double t = lo;
      lo = hi;
      hi = t;
    }
    double c = dt;
    if (c < lo) c = lo;                      // maximum(dt, lo)
    if (c > hi) c = hi;                      // minimum(., hi)
    dt_raw = c;
  }
  double m = dt * factor;
  if (dt_raw < m) m = dt_raw;
  const double cap = 0.005 * ctld;
  if (cap < m) m = cap;
  if (t_cfl < m) m = t_cfl;
  return m;
}

// Block-wide max of non-negative values (NaN already filtered by the caller).
template <int NT>
__device__ __forceinline__ double block_max(double v, double *red) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  const int lane = threadIdx.x & 31, warp = (threadIdx.y * blockDim.x + threadIdx.x) >> 5;
  if (lane == 0) red[warp] = v;
  __syncthreads();
  if (warp == 0) {
    v = (lane < NT / 32) ? red[lane] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  }
  return v;
}

// Locality key of the table cell of a composition, for ordering points by
// cell: a hash of the four cell indices floor(u_a), u = x / resolution,
// estimated in FP32 (only the order of work depends on it, never a value).
// The 16 cells of any 2x2x2x2 block of cells get distinct keys.
__device__ __forceinline__ int cell_hash_u(const float u[S]) {
  const unsigned w[S] = {41u, 13u, 5u, 1u};
  unsigned h = 0;
#pragma unroll
  for (int a = 0; a < S; ++a) h += (unsigned)(int)floorf(u[a]) * w[a];
  return (int)(h & 255u);
}

__device__ __forceinline__ int cell_hash(const double x[S], float inv_step) {
  float u[S];
#pragma unroll
  for (int a = 0; a < S; ++a) u[a] = (float)x[a] * inv_step;
  return cell_hash_u(u);
}

// Block-wide exclusive prefix sum of bins[0..NB) by all NT threads of the
// block (consecutive bins per thread); wsum holds NT/32 + 1 ints.  Returns
// the total and ends with a barrier.
template <int NB, int NT>
__device__ __forceinline__ int block_exclusive_scan(int *bins, int *wsum, int tid) {
  constexpr int BPT = (NB + NT - 1) / NT;
  const int lane = tid & 31, w = tid >> 5;
  int loc[BPT];
  int v = 0;
#pragma unroll
  for (int j = 0; j < BPT; ++j) {
    const int b = tid * BPT + j;
    loc[j] = b < NB ? bins[b] : 0;
    v += loc[j];
  }
  int inc = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int t = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += t;
  }
  if (lane == 31) wsum[w] = inc;
  __syncthreads();
  if (w == 0) {
    const int t = lane < NT / 32 ? wsum[lane] : 0;
    int sc = t;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int u = __shfl_up_sync(0xffffffffu, sc, o);
      if (lane >= o) sc += u;
    }
    if (lane < NT / 32) wsum[lane] = sc - t;
    if (lane == NT / 32 - 1) wsum[NT / 32] = sc;
  }
  __syncthreads();
  int base = inc - v + wsum[w];
#pragma unroll
  for (int j = 0; j < BPT; ++j) {
    const int b = tid * BPT + j;
    if (b < NB) bins[b] = base;
    base += loc[j];
  }
  const int total = wsum[NT / 32];
  __syncthreads();
  return total;
}

// Wait for the previous kernel of the stream (and its memory) when this
// kernel was launched with programmatic stream serialization; a no-op
// otherwise.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

}  // namespace pf5d
