// pf5d_diag.cuh -- save-step diagnostics of the plain FP64 stepper
// (examples/simulate.py:299-354): reductions over the field before and after
// the update of one step.  Each kernel writes one row of partial results per
// block; the host adds the rows in block order (FP64, fixed order).
#pragma once

#include "pf5d_device.cuh"

namespace pf5d {

constexpr int kDiagThreads = 256;
constexpr int kDiagBlocks = 592;           // 4 x 148 SMs
constexpr int kDiagPre = 3 * S;            // net, max |dX/dt|, total flux
constexpr int kDiagPost = 3 * S + 2;       // mass, min, max, max sum_s X_s, sum X . kappa lap X
constexpr int kDiagVar = S;                // sum (X - mean)^2

struct DiagGeom {
  int nz, ny, nx, dim;
  int64_t npts;
  double inv_dx, inv_dx2;
  double kappa[S];
};

// Linear index of the neighbour of point g = (z, y, x) one step along spatial
// axis `a` (0 = first axis of the field) in direction d = +1 / -1 (periodic).
__device__ __forceinline__ int64_t diag_neighbour(const DiagGeom &G, int64_t g, int a, int d) {
  const int x = (int)(g % G.nx);
  const int64_t r = g / G.nx;
  const int y = (int)(r % G.ny);
  const int z = (int)(r / G.ny);
  // spatial axis a of a dim-D field maps onto (z, y, x) from the back
  const int slot = 3 - G.dim + a;          // 0 = z, 1 = y, 2 = x
  int xx = x, yy = y, zz = z;
  if (slot == 2) xx = d > 0 ? (x + 1 == G.nx ? 0 : x + 1) : (x == 0 ? G.nx - 1 : x - 1);
  else if (slot == 1) yy = d > 0 ? (y + 1 == G.ny ? 0 : y + 1) : (y == 0 ? G.ny - 1 : y - 1);
  else zz = d > 0 ? (z + 1 == G.nz ? 0 : z + 1) : (z == 0 ? G.nz - 1 : z - 1);
  return ((int64_t)zz * G.ny + yy) * G.nx + xx;
}

__device__ __forceinline__ void diag_load4(const double *X, int64_t g, double v[S]) {
  const double2 a = __ldg(reinterpret_cast<const double2 *>(X + 4 * g));
  const double2 b = __ldg(reinterpret_cast<const double2 *>(X + 4 * g) + 1);
  v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
}

// Block reduction of K values per thread (sum, or max where is_max[k]);
// thread 0 writes the block's row.
template <int K>
__device__ __forceinline__ void diag_block_row(double v[K], const bool is_max[K], double *row) {
  __shared__ double red[kDiagThreads / 32][K];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < K; ++k) {
    double x = v[k];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const double y = __shfl_xor_sync(0xffffffffu, x, o);
      x = is_max[k] ? fmax(x, y) : x + y;
    }
    if (lane == 0) red[w][k] = x;
  }
  __syncthreads();
  if (threadIdx.x < K) {
    const int k = threadIdx.x;
    double x = red[0][k];
    for (int i = 1; i < kDiagThreads / 32; ++i) x = is_max[k] ? fmax(x, red[i][k]) : x + red[i][k];
    row[k] = x;
  }
}

// Before the update: net = sum dX/dt, max |dX/dt| per component, and the
// total flux sum over points and axes of (flux_p - flux_m), with
// flux_p / flux_m the face fluxes of each point towards its +/- neighbour
// from the forward / backward mu gradients (operators.py:88-123 gradients,
// fluxes.py:6-125 compute_fluxes).  mm: mu_1..4 then M_Fe, M_1..4, SoA.
__global__ void __launch_bounds__(kDiagThreads) k_diag_pre(DiagGeom G, const double *X,
                                                           const double *dX, const double *mm,
                                                           double *partial) {
  double v[kDiagPre];
  bool is_max[kDiagPre];
#pragma unroll
  for (int k = 0; k < kDiagPre; ++k) {
    v[k] = 0.0;
    is_max[k] = (k >= S && k < 2 * S);
  }
  for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < G.npts;
       g += (int64_t)gridDim.x * blockDim.x) {
    double d[S], xc[S], mc[NM], muc[S];
    diag_load4(dX, g, d);
    diag_load4(X, g, xc);
#pragma unroll
    for (int c = 0; c < S; ++c) {
      v[c] = v[c] + d[c];
      v[S + c] = fmax(v[S + c], fabs(d[c]));
      muc[c] = mm[c * G.npts + g];
    }
#pragma unroll
    for (int c = 0; c < NM; ++c) mc[c] = mm[(S + c) * G.npts + g];
    for (int a = 0; a < G.dim; ++a) {
      const int64_t gp = diag_neighbour(G, g, a, +1), gm = diag_neighbour(G, g, a, -1);
      double xn[S], mn[NM], grad[S], fp[S], fm[S];
      diag_load4(X, gp, xn);
#pragma unroll
      for (int c = 0; c < NM; ++c) mn[c] = mm[(S + c) * G.npts + gp];
#pragma unroll
      for (int c = 0; c < S; ++c) grad[c] = (mm[c * G.npts + gp] - muc[c]) * G.inv_dx;
      face_flux(xc, mc, xn, mn, grad, fp);
      diag_load4(X, gm, xn);
#pragma unroll
      for (int c = 0; c < NM; ++c) mn[c] = mm[(S + c) * G.npts + gm];
#pragma unroll
      for (int c = 0; c < S; ++c) grad[c] = (muc[c] - mm[c * G.npts + gm]) * G.inv_dx;
      face_flux(xc, mc, xn, mn, grad, fm);
#pragma unroll
      for (int c = 0; c < S; ++c) v[2 * S + c] = v[2 * S + c] + (fp[c] - fm[c]);
    }
  }
  diag_block_row<kDiagPre>(v, is_max, partial + blockIdx.x * kDiagPre);
}

// After the update: mass = sum X, min / max per component, max over points
// of sum_s X_s (for comp_fe_min), and sum X . (kappa lap X) (for f_grad;
// Laplacian as operators.py:33-76, then scaled by kappa per component).
__global__ void __launch_bounds__(kDiagThreads) k_diag_post(DiagGeom G, const double *X,
                                                            double *partial) {
  double v[kDiagPost];
  bool is_max[kDiagPost];
#pragma unroll
  for (int k = 0; k < kDiagPost; ++k) is_max[k] = (k >= 2 * S && k < 3 * S + 1) || (k >= S && k < 2 * S);
#pragma unroll
  for (int c = 0; c < S; ++c) {
    v[c] = 0.0;
    v[S + c] = -INFINITY;           // stored negated: max of -X is -min X
    v[2 * S + c] = -INFINITY;
  }
  v[3 * S] = -INFINITY;
  v[3 * S + 1] = 0.0;
  for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < G.npts;
       g += (int64_t)gridDim.x * blockDim.x) {
    double xc[S], lap[S], n0[S], n1[S];
    diag_load4(X, g, xc);
    // Laplacian: +axis0, -axis0, +axis1, -axis1, ... then - 2*dim*c
    for (int c = 0; c < S; ++c) lap[c] = 0.0;
    for (int a = 0; a < G.dim; ++a) {
      diag_load4(X, diag_neighbour(G, g, a, +1), n0);
      diag_load4(X, diag_neighbour(G, g, a, -1), n1);
#pragma unroll
      for (int c = 0; c < S; ++c) lap[c] = a == 0 ? n0[c] + n1[c] : (lap[c] + n0[c]) + n1[c];
    }
    const double w = G.dim == 1 ? 2.0 : (G.dim == 2 ? 4.0 : 6.0);
    double sum = 0.0, fg = 0.0;
#pragma unroll
    for (int c = 0; c < S; ++c) {
      const double l = ((lap[c] - w * xc[c]) * G.inv_dx2) * G.kappa[c];
      v[c] = v[c] + xc[c];
      v[S + c] = fmax(v[S + c], -xc[c]);
      v[2 * S + c] = fmax(v[2 * S + c], xc[c]);
      sum = sum + xc[c];
      fg = fg + xc[c] * l;
    }
    v[3 * S] = fmax(v[3 * S], sum);
    v[3 * S + 1] = v[3 * S + 1] + fg;
  }
  diag_block_row<kDiagPost>(v, is_max, partial + blockIdx.x * kDiagPost);
}

// Second pass of the variance: sum (X - mean)^2 per component.
__global__ void __launch_bounds__(kDiagThreads) k_diag_var(DiagGeom G, const double *X,
                                                           const double *mean, double *partial) {
  double v[kDiagVar];
  bool is_max[kDiagVar];
  double m[S];
#pragma unroll
  for (int c = 0; c < S; ++c) {
    v[c] = 0.0;
    is_max[c] = false;
    m[c] = mean[c];
  }
  for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < G.npts;
       g += (int64_t)gridDim.x * blockDim.x) {
    double xc[S];
    diag_load4(X, g, xc);
#pragma unroll
    for (int c = 0; c < S; ++c) {
      const double e = xc[c] - m[c];
      v[c] = v[c] + e * e;
    }
  }
  diag_block_row<kDiagVar>(v, is_max, partial + blockIdx.x * kDiagVar);
}

}  // namespace pf5d
