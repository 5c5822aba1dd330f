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
//        - dX/dt written once; block max |dX/dt| folded into a device
//          accumulator; the last block to finish evaluates the adaptive dt
//          rule and advances dt, time and the step counter on the device.
//   5. k_update_step: X += dX*dt; clamp; s for the next step; every
//      oob_interval steps the out_of_bounds test, which halts the stepper
//      (every later kernel returns at entry) on a hard violation.
//
// Every FP64 operation follows the reference's order; the unit is compiled
// with -fmad=false, so apart from the FFT (cuFFT vs pocketfft rounding) the
// trajectory equals the reference's bit for bit.
#include <algorithm>
#include <map>
#include <vector>

#include "pf5d_device.cuh"
#include "pf5d_fft.h"

namespace pf5d {

struct StepState {
  double dt;
  double time;
  double xdotmax;      // max |dX/dt| of the last rate evaluation
  double xacc;         // running max of the current evaluation (bit-wise atomicMax)
  unsigned blocks_done;
  unsigned flags;      // PF5D_FLAG_* accumulated
  unsigned halt;       // non-zero: every step kernel returns at entry
  unsigned pad;
  long long step;      // completed steps
};

struct RateParams {
  int nz, ny, nx;              // axis 0 (march), axis 1 (3D only, else 1), last axis
  const double *X;
  const double *sp;            // s' (already scaled by 1/N) or nullptr
  double *dX;
  Table T;
  Vec4 kappa, lvec;
  double inv_dx, inv_dx2;
  double ctld, t_cfl, lower, upper, factor;
  int adaptive;
  StepState *st;
};

// ------------------------------------------------------------------------
// Shared pieces of the rate kernels
// ------------------------------------------------------------------------

// chemical potential and mobility at one point (examples/simulate.py:242-258).
__device__ __forceinline__ void chem_point(const RateParams &P, const double x[S],
                                           const double lap[S], double spv, double mu[S],
                                           double M[NM], unsigned *flags) {
  double v[NP];
  interp_point(P.T, x, v, flags);
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

// Fold this thread's max |dX/dt| into the block, then into the device
// accumulator; the last block of the launch runs the dt controller.
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
    StepState *st = P.st;
    atomic_max_nonneg(&st->xacc, m);
    __threadfence();
    const unsigned total = gridDim.x * gridDim.y * gridDim.z;
    const unsigned prev = atomicAdd(&st->blocks_done, 1u);
    if (prev == total - 1) {
      __threadfence();
      const double xmax = __longlong_as_double(
          (long long)atomicAdd(reinterpret_cast<unsigned long long *>(&st->xacc), 0ULL));
      double dt = st->dt;
      if (P.adaptive) dt = adaptive_dt(dt, xmax, P.ctld, P.t_cfl, P.lower, P.upper, P.factor);
      st->dt = dt;
      st->time = st->time + dt;
      st->xdotmax = xmax;
      st->step = st->step + 1;
      st->xacc = 0.0;
      st->blocks_done = 0;
    }
  }
}

// ------------------------------------------------------------------------
// 2D / 3D marching kernel
// ------------------------------------------------------------------------
// Plane = TY x TX tile of (axis 1, last axis) for DIM 3, a TX row segment of
// the last axis for DIM 2 (TY = 1).  X ring: 3 planes with a 2-cell halo
// (HY x HX).  mu/M ring: 2 planes with a 1-cell halo (MY x MX), 9 values per
// point (mu 0..3, M 4..8).  Face buffers hold the tile's +x / +y fluxes and
// the tile-boundary -x / -y fluxes.
template <int DIM, int TX, int TY>
struct MarchGeom {
  static constexpr int HX = TX + 4, HY = DIM == 3 ? TY + 4 : 1, PX = HX * HY;
  static constexpr int MX = TX + 2, MY = DIM == 3 ? TY + 2 : 1, PM = MX * MY;
  static constexpr int NT = TX * TY;
  static constexpr int FXN = TY * (TX + 1), FYN = DIM == 3 ? (TY + 1) * TX : 0;
  static constexpr size_t smem_doubles =
      3 * S * PX + 2 * NP * PM + S * FXN + S * FYN + (NT + 31) / 32;
  static constexpr size_t smem_bytes = smem_doubles * sizeof(double);
};

template <int DIM, int TX, int TY>
__global__ void __launch_bounds__(TX * TY, DIM == 3 ? 2 : 4)
    k_rate_march(RateParams P, int zc) {
  using G = MarchGeom<DIM, TX, TY>;
  if (P.st->halt) return;
  extern __shared__ double sm[];
  double *Xs = sm;                                  // [3][S][PX]
  double *Ms = Xs + 3 * S * G::PX;                  // [2][NP][PM]
  double *Fx = Ms + 2 * NP * G::PM;                 // [S][TY][TX+1]
  double *Fy = Fx + S * G::FXN;                     // [S][TY+1][TX]
  double *red = Fy + S * G::FYN;

  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
  const int x0 = blockIdx.x * TX, y0 = (DIM == 3) ? blockIdx.y * TY : 0;
  const int zb = blockIdx.z * zc;
  const int ze = min(zb + zc, P.nz);
  unsigned flags = 0;

  auto xplane = [&](int z) { return Xs + ((z - zb + 3) % 3) * S * G::PX; };
  auto mplane = [&](int z) { return Ms + ((z - zb + 2) & 1) * NP * G::PM; };

  auto load_x = [&](int z) {
    double *dst = xplane(z);
    const int zw = wrap_any(z, P.nz);
    for (int pos = tid; pos < G::PX; pos += G::NT) {
      const int hx = pos % G::HX, hy = pos / G::HX;
      const int gx = wrap_any(x0 + hx - 2, P.nx);
      const int gy = (DIM == 3) ? wrap_any(y0 + hy - 2, P.ny) : 0;
      const int64_t g = ((int64_t)zw * P.ny + gy) * P.nx + gx;
      const double2 a = __ldg(reinterpret_cast<const double2 *>(P.X + 4 * g));
      const double2 b = __ldg(reinterpret_cast<const double2 *>(P.X + 4 * g) + 1);
      dst[0 * G::PX + pos] = a.x;
      dst[1 * G::PX + pos] = a.y;
      dst[2 * G::PX + pos] = b.x;
      dst[3 * G::PX + pos] = b.y;
    }
  };

  // mu/M of plane z at muM positions; interior_only: tile positions only.
  auto compute_mu = [&](int z, bool interior_only) {
    const double *Xm = xplane(z - 1), *X0p = xplane(z), *Xp = xplane(z + 1);
    double *dst = mplane(z);
    const int zw = wrap_any(z, P.nz);
    for (int pos = tid; pos < G::PM; pos += G::NT) {
      const int mx = pos % G::MX, my = pos / G::MX;
      const bool edge_x = (mx == 0 || mx == G::MX - 1);
      const bool edge_y = (DIM == 3) && (my == 0 || my == G::MY - 1);
      if (interior_only ? (edge_x || edge_y) : (edge_x && edge_y)) continue;
      const int px = (DIM == 3) ? (my + 1) * G::HX + (mx + 1) : (mx + 1);
      double x[S], lap[S];
#pragma unroll
      for (int c = 0; c < S; ++c) {
        const double *q = X0p + c * G::PX;
        x[c] = q[px];
        double a = Xp[c * G::PX + px] + Xm[c * G::PX + px];
        if (DIM == 3) {
          a = a + q[px + G::HX];
          a = a + q[px - G::HX];
        }
        a = a + q[px + 1];
        a = a + q[px - 1];
        lap[c] = (a - (DIM == 3 ? 6.0 : 4.0) * x[c]) * P.inv_dx2;
      }
      double spv = 0.0;
      if (P.sp) {
        const int gx = wrap_any(x0 + mx - 1, P.nx);
        const int gy = (DIM == 3) ? wrap_any(y0 + my - 1, P.ny) : 0;
        spv = __ldg(P.sp + ((int64_t)zw * P.ny + gy) * P.nx + gx);
      }
      double mu[S], M[NM];
      chem_point(P, x, lap, spv, mu, M, &flags);
#pragma unroll
      for (int c = 0; c < S; ++c) dst[c * G::PM + pos] = mu[c];
#pragma unroll
      for (int c = 0; c < NM; ++c) dst[(S + c) * G::PM + pos] = M[c];
    }
  };

  // flux through the face between (plane zl, X pos pl, muM pos ql) and (zh, ph, qh).
  auto face = [&](int zl, int pl, int ql, int zh, int ph, int qh, double J[S]) {
    const double *XL = xplane(zl), *XH = xplane(zh);
    const double *ML = mplane(zl), *MH = mplane(zh);
    double Xc[S], Xn[S], Mc[NM], Mn[NM], g[S];
#pragma unroll
    for (int c = 0; c < S; ++c) {
      Xc[c] = XL[c * G::PX + pl];
      Xn[c] = XH[c * G::PX + ph];
      g[c] = (MH[c * G::PM + qh] - ML[c * G::PM + ql]) * P.inv_dx;
    }
#pragma unroll
    for (int c = 0; c < NM; ++c) {
      Mc[c] = ML[(S + c) * G::PM + ql];
      Mn[c] = MH[(S + c) * G::PM + qh];
    }
    face_flux(Xc, Mc, Xn, Mn, g, J);
  };

  const int pX = (DIM == 3) ? (ty + 2) * G::HX + (tx + 2) : (tx + 2);
  const int pM = (DIM == 3) ? (ty + 1) * G::MX + (tx + 1) : (tx + 1);
  const bool in_tile = (x0 + tx < P.nx) && (DIM == 2 || y0 + ty < P.ny);

  // Prologue: X planes zb-2..zb+1, mu of zb-1 (tile) and zb (tile + halo),
  // then the -axis0 face of plane zb.
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
  double Jm[S];
  face(zb - 1, pX, pM, zb, pX, pM, Jm);

  double vmax = 0.0;
  for (int z = zb; z < ze; ++z) {
    __syncthreads();
    load_x(z + 2);
    __syncthreads();
    compute_mu(z + 1, false);
    __syncthreads();
    double Jz[S], J[S];
    face(z, pX, pM, z + 1, pX, pM, Jz);                          // +axis0
    face(z, pX, pM, z, pX + 1, pM + 1, J);                       // +x
#pragma unroll
    for (int c = 0; c < S; ++c) Fx[c * G::FXN + ty * (TX + 1) + tx + 1] = J[c];
    if (DIM == 3) {
      face(z, pX, pM, z, pX + G::HX, pM + G::MX, J);             // +y
#pragma unroll
      for (int c = 0; c < S; ++c) Fy[c * G::FYN + (ty + 1) * TX + tx] = J[c];
    }
    // tile-boundary faces: -x of column 0 (threads 0..TY-1), -y of row 0.
    if (tid < TY) {
      const int r = tid;
      const int bx = (DIM == 3) ? (r + 2) * G::HX + 2 : 2;
      const int bm = (DIM == 3) ? (r + 1) * G::MX + 1 : 1;
      face(z, bx - 1, bm - 1, z, bx, bm, J);
#pragma unroll
      for (int c = 0; c < S; ++c) Fx[c * G::FXN + r * (TX + 1)] = J[c];
    }
    if (DIM == 3 && tid >= 32 && tid < 32 + TX) {
      const int col = tid - 32;
      const int bx = 2 * G::HX + col + 2, bm = G::MX + col + 1;
      face(z, bx - G::HX, bm - G::MX, z, bx, bm, J);
#pragma unroll
      for (int c = 0; c < S; ++c) Fy[c * G::FYN + col] = J[c];
    }
    __syncthreads();
    if (in_tile) {
      double out[S];
#pragma unroll
      for (int c = 0; c < S; ++c) {
        double a = Jz[c] - Jm[c];
        if (DIM == 3) {
          a = a + Fy[c * G::FYN + (ty + 1) * TX + tx];
          a = a - Fy[c * G::FYN + ty * TX + tx];
        }
        a = a + Fx[c * G::FXN + ty * (TX + 1) + tx + 1];
        a = a - Fx[c * G::FXN + ty * (TX + 1) + tx];
        out[c] = a * P.inv_dx;
        const double v = fabs(out[c]);
        if (v > vmax) vmax = v;
      }
      const int64_t g = ((int64_t)z * P.ny + (y0 + ty)) * P.nx + (x0 + tx);
      double2 *o = reinterpret_cast<double2 *>(P.dX + 4 * g);
      o[0] = make_double2(out[0], out[1]);
      o[1] = make_double2(out[2], out[3]);
    }
#pragma unroll
    for (int c = 0; c < S; ++c) Jm[c] = Jz[c];
  }
  if (flags) atomicOr(&P.st->flags, flags);
  finish_rate(P, vmax, red);
}

// ------------------------------------------------------------------------
// 1D kernel: a tile of TX points with halos, no marching.
// ------------------------------------------------------------------------
template <int TX>
__global__ void __launch_bounds__(TX) k_rate_1d(RateParams P) {
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
    chem_point(P, x, lap, spv, mu, M, &flags);
#pragma unroll
    for (int c = 0; c < S; ++c) Ms[c][pos] = mu[c];
#pragma unroll
    for (int c = 0; c < NM; ++c) Ms[S + c][pos] = M[c];
  }
  __syncthreads();
  auto face = [&](int ml, double J[S]) {   // face between muM pos ml and ml+1
    double Xc[S], Xn[S], Mc[NM], Mn[NM], g[S];
#pragma unroll
    for (int c = 0; c < S; ++c) {
      Xc[c] = Xs[c][ml + 1];
      Xn[c] = Xs[c][ml + 2];
      g[c] = (Ms[c][ml + 1] - Ms[c][ml]) * P.inv_dx;
    }
#pragma unroll
    for (int c = 0; c < NM; ++c) {
      Mc[c] = Ms[S + c][ml];
      Mn[c] = Ms[S + c][ml + 1];
    }
    face_flux(Xc, Mc, Xn, Mn, g, J);
  };
  double J[S];
  face(tx + 1, J);
#pragma unroll
  for (int c = 0; c < S; ++c) Fx[c][tx + 1] = J[c];
  if (tx == 0) {
    face(0, J);
#pragma unroll
    for (int c = 0; c < S; ++c) Fx[c][0] = J[c];
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
  if (flags) atomicOr(&P.st->flags, flags);
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

}  // namespace pf5d

using namespace pf5d;

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
};

namespace {

constexpr int kTX3 = 32, kTY3 = 8;   // 3D plane tile
constexpr int kTX2 = 64;             // 2D row segment
constexpr int kTX1 = 128;            // 1D tile
constexpr int kGraphSteps = 50;      // steps per captured graph

pf5d_status configure_rate(pf5d_stepper *h) {
  const int dim = h->d.dim;
  const int nsm = sm_count();
  if (dim == 1) {
    h->rate_block = dim3(kTX1);
    h->rate_grid = dim3((unsigned)((h->rp.nx + kTX1 - 1) / kTX1));
    h->rate_smem = 0;
    return PF5D_OK;
  }
  int tiles;
  if (dim == 2) {
    using G = MarchGeom<2, kTX2, 1>;
    h->rate_block = dim3(kTX2, 1);
    tiles = (h->rp.nx + kTX2 - 1) / kTX2;
    h->rate_smem = G::smem_bytes;
    PF5D_CUDA(cudaFuncSetAttribute(k_rate_march<2, kTX2, 1>,
                                   cudaFuncAttributeMaxDynamicSharedMemorySize, (int)G::smem_bytes));
  } else {
    using G = MarchGeom<3, kTX3, kTY3>;
    h->rate_block = dim3(kTX3, kTY3);
    tiles = ((h->rp.nx + kTX3 - 1) / kTX3) * ((h->rp.ny + kTY3 - 1) / kTY3);
    h->rate_smem = G::smem_bytes;
    PF5D_CUDA(cudaFuncSetAttribute(k_rate_march<3, kTX3, kTY3>,
                                   cudaFuncAttributeMaxDynamicSharedMemorySize, (int)G::smem_bytes));
  }
  // Chunk length along axis 0: aim for ~8 blocks per SM, at least 4 planes.
  const int64_t target = (int64_t)nsm * 8;
  int64_t zc = ((int64_t)tiles * h->rp.nz + target - 1) / target;
  zc = std::max<int64_t>(dim == 2 ? 8 : 4, std::min<int64_t>(zc, 64));
  zc = std::min<int64_t>(zc, h->rp.nz);
  h->zc = (int)zc;
  const unsigned nzb = (unsigned)((h->rp.nz + zc - 1) / zc);
  if (dim == 2)
    h->rate_grid = dim3((unsigned)tiles, 1, nzb);
  else
    h->rate_grid = dim3((unsigned)((h->rp.nx + kTX3 - 1) / kTX3),
                        (unsigned)((h->rp.ny + kTY3 - 1) / kTY3), nzb);
  return PF5D_OK;
}

pf5d_status launch_rate(pf5d_stepper *h, cudaStream_t s) {
  switch (h->d.dim) {
    case 1: k_rate_1d<kTX1><<<h->rate_grid, h->rate_block, 0, s>>>(h->rp); break;
    case 2:
      k_rate_march<2, kTX2, 1><<<h->rate_grid, h->rate_block, h->rate_smem, s>>>(h->rp, h->zc);
      break;
    default:
      k_rate_march<3, kTX3, kTY3><<<h->rate_grid, h->rate_block, h->rate_smem, s>>>(h->rp, h->zc);
  }
  PF5D_LAUNCHED();
  return PF5D_OK;
}

pf5d_status enqueue_step(pf5d_stepper *h, cudaStream_t s) {
  pf5d_status st;
  if (h->d.elastic) {
    if ((st = fft_forward(&h->fft, h->s, h->k, s)) != PF5D_OK) return st;
    if ((st = launch_bmul(h->k, h->bk, h->fft.nk, &h->st->halt, s)) != PF5D_OK) return st;
    if ((st = fft_inverse(&h->fft, h->k, h->s, s)) != PF5D_OK) return st;
  }
  if ((st = launch_rate(h, s)) != PF5D_OK) return st;
  k_update_step<<<grid_for(h->npts, 256, 4), 256, 0, s>>>(h->up);
  PF5D_LAUNCHED();
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
  if (desc->elastic) {
    if ((st = fft_create(desc->dim, h->shape, &h->fft)) != PF5D_OK) return fail(st);
    if ((st = upload_bk_scaled(desc->bk, h->fft.nk, npts, &h->bk)) != PF5D_OK) return fail(st);
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
    P.nz = (int)h->shape[0]; P.ny = 1; P.nx = (int)h->shape[1];
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
  P.T.exact_d2 = (1.99 * desc->resolution) * (1.99 * desc->resolution);
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
  if ((st = configure_rate(h)) != PF5D_OK) return fail(st);
  if ((st = pf5d_stepper_reset(h, desc->dt0, 0.0, stream)) != PF5D_OK) return fail(st);
  (void)s;
  *out = h;
  return PF5D_OK;
}

pf5d_status pf5d_stepper_reset(pf5d_stepper *h, double dt, double time, void *stream) {
  PF5D_REQUIRE(h, PF5D_ERR_ARG, "null stepper");
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

double *pf5d_stepper_rate(pf5d_stepper *h) { return h ? h->dX : nullptr; }

pf5d_status pf5d_stepper_launch_stage(pf5d_stepper *h, int32_t stage, void *stream) {
  PF5D_REQUIRE(h, PF5D_ERR_ARG, "null stepper");
  cudaStream_t s = as_stream(stream);
  switch (stage) {
    case PF5D_STAGE_RATE:
      return launch_rate(h, s);
    case PF5D_STAGE_UPDATE:
      k_update_step<<<grid_for(h->npts, 256, 4), 256, 0, s>>>(h->up);
      PF5D_LAUNCHED();
      return PF5D_OK;
    case PF5D_STAGE_FFT_FWD:
      PF5D_REQUIRE(h->d.elastic, PF5D_ERR_ARG, "elasticity is off");
      return fft_forward(&h->fft, h->s, h->k, s);
    case PF5D_STAGE_BMUL:
      PF5D_REQUIRE(h->d.elastic, PF5D_ERR_ARG, "elasticity is off");
      return launch_bmul(h->k, h->bk, h->fft.nk, &h->st->halt, s);
    case PF5D_STAGE_FFT_INV:
      PF5D_REQUIRE(h->d.elastic, PF5D_ERR_ARG, "elasticity is off");
      return fft_inverse(&h->fft, h->k, h->s, s);
    default:
      set_error("unknown stage %d", stage);
      return PF5D_ERR_ARG;
  }
}

pf5d_status pf5d_stepper_destroy(pf5d_stepper *h) {
  if (!h) return PF5D_OK;
  for (auto &kv : h->graphs) cudaGraphExecDestroy(kv.second);
  fft_destroy(&h->fft);
  cudaFree(h->dX);
  cudaFree(h->s);
  cudaFree(h->k);
  cudaFree(h->bk);
  cudaFree(h->st);
  if (h->cap) cudaStreamDestroy(h->cap);
  delete h;
  return PF5D_OK;
}

}  // extern "C"
