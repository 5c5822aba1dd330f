// pf5d_fp32c.cuh -- device numerics of the FP32-compensated form, shared by
// the single-solve stepper (precision.cu) and the batched stepper
// (batch.cu): step state, FP32 table view and per-solve parameters, cell /
// interpolation / face-flux routines, the per-plane mu evaluation with the
// shared table window, and the compensated-update helpers.
#pragma once


#include <cufft.h>

#include "pf5d_device.cuh"
#include "pf5d_tiles.cuh"
#include "pf5d_window.cuh"

namespace pf5d {

struct StepState32 {
  double dt;
  double time;
  double xdotmax;
  unsigned flags;
  unsigned halt;
  long long step;
};

constexpr int kStride32 = 12;   // floats per FP32 table node (9 props + 3 pad = 48 bytes)
// Rows of a mu/M array in shared memory: mu_1..4, M_Fe, M_1..4 and the
// point's FP64-formed closure X_Fe = (1 - sum X0) - sum D, rounded to FP32.
constexpr int NPM = NP + 1;

struct Table32 {
  const float *grid;
  const double *coord;
  int n;
  int stride;
  double inv_step, threshold, max_nn_dist;
  float inv_step_f;
  int ib[S];          // floor(X0_d / res)
  float fb[S];        // X0_d / res - floor(X0_d / res)
  double x0[S];
  double sum_x0;
};

struct Rate32 {
  int nz, ny, nx;
  const float4 *D;     // hi part of X - X0
  const float *sp;     // s' scaled by 1/N, or nullptr
  float4 *dX;
  Table32 T;
  float kappa[S], lvec[S], x0f[S];
  double c_fe;         // 1 - sum X0
  float flux_scale;    // 0.5 / dx^2: divergence scale of the unscaled face fluxes
  float inv_dx2;
  double ctld, t_cfl, lower, upper, factor;
  int adaptive;
  StepState32 *st;
  double *partial;     // block maxima of |dX/dt| of the last rate launch
  // split rate buffers, one entry per point: mu_1..4; M_1..4; (M_Fe, X_Fe)
  float4 *mm_mu, *mm_m;
  float2 *mm_f;
  int64_t npts;
};

// ------------------------------------------------------------------------
// Device numerics
// ------------------------------------------------------------------------

// FP32 Laplacian of one component: the N neighbour values in the
// reference's order (+axis0, -axis0, +axis1, ...), minus N * centre, times
// 1/dx^2 (operators.py:33-76).  Every operation is separately rounded, so
// the fused, split and batched kernels agree bit for bit.
template <int N>
__device__ __forceinline__ float lap32(const float nb[N], float c, float inv_dx2) {
  float sum = nb[0];
#pragma unroll
  for (int i = 1; i < N; ++i) sum = __fadd_rn(sum, nb[i]);
  return __fmul_rn(__fsub_rn(sum, __fmul_rn((float)N, c)), inv_dx2);
}

// FP64 sum of the deviation d = X - X0 (left to right): the linear-region
// test and the closure X_Fe = (1 - sum X0) - sum d both use it.
__device__ __forceinline__ double dsum32(const float d[S]) {
  return (((double)d[0] + (double)d[1]) + (double)d[2]) + (double)d[3];
}

// Table cell and fractional coordinates of X = X0 + d (interpolation.py:103-121
// clamping); sd = dsum32(d).  Returns false when the point is outside the
// linear region (sum X > 1 - 4 res - 1e-9, tested in FP64) and takes the
// nearest-row path.
__device__ __forceinline__ bool cell32(const Table32 &T, const float d[S], double sd, int ii[S],
                                       float tt[S]) {
  if (!(T.sum_x0 + sd <= T.threshold)) return false;
#pragma unroll
  for (int a = 0; a < S; ++a) {
    const float v = fmaf(d[a], T.inv_step_f, T.fb[a]);
    const float k = floorf(v);
    int i = T.ib[a] + (int)k;
    float t = v - k;
    if (i < 0) {
      i = 0;
      t = 0.f;
    } else if (i > T.n - 2) {
      i = T.n - 2;
      t = 1.f;
    }
    ii[a] = i;
    tt[a] = t;
  }
  return true;
}

// Corner weights of the quadrilinear interpolation as two pair products:
// corner c = b0 b1 b2 b3 (binary) has weight wa[b0 b1] * wb[b2 b3], where
// wa = {q0 q1, q0 t1, t0 q1, t0 t1}, wb likewise for axes 2, 3 (q = 1 - t).
struct Weights32 {
  float wa[4], wb[4];
};

__device__ __forceinline__ Weights32 weights32(const float tt[S]) {
  const float q0 = 1.f - tt[0], q1 = 1.f - tt[1], q2 = 1.f - tt[2], q3 = 1.f - tt[3];
  Weights32 w;
  w.wa[0] = q0 * q1;
  w.wa[1] = q0 * tt[1];
  w.wa[2] = tt[0] * q1;
  w.wa[3] = tt[0] * tt[1];
  w.wb[0] = q2 * q3;
  w.wb[1] = q2 * tt[3];
  w.wb[2] = tt[2] * q3;
  w.wb[3] = tt[2] * tt[3];
  return w;
}

// One corner's contribution: out[p] = w v[p] for the first corner, else
// fma(w, v[p], out[p]) -- corners in order c = 0..15 in every kernel.
__device__ __forceinline__ void corner_acc32(int c, float w, const float4 &a, const float4 &b,
                                             const float4 &e, float out[NP]) {
  const float v[NP] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w, e.x};
#pragma unroll
  for (int p = 0; p < NP; ++p) out[p] = (c == 0) ? w * v[p] : fmaf(w, v[p], out[p]);
}

// Quadrilinear interpolation of the 9 props from 16 corner nodes laid out
// with node strides (s0, s1, s2, s3) in float4 units from `base` (global
// table or shared window; 3 float4 per node).
__device__ __forceinline__ void interp_nodes32(const float4 *base, int s0, int s1, int s2, int s3,
                                               const float tt[S], float out[NP]) {
  const Weights32 W = weights32(tt);
#pragma unroll
  for (int c = 0; c < 16; ++c) {
    const int b0 = (c >> 3) & 1, b1 = (c >> 2) & 1, b2 = (c >> 1) & 1, b3 = c & 1;
    const float w = W.wa[c >> 2] * W.wb[c & 3];
    const float4 *node = base + b0 * s0 + b1 * s1 + b2 * s2 + b3 * s3;
    corner_acc32(c, w, node[0], node[1], node[2], out);
  }
}

// Nearest table row (the fallback outside the linear region) of X0 + d.
__device__ __forceinline__ void nearest_row32(const Table32 &T, const float d[S], float out[NP],
                                              unsigned *flags) {
  const NearestNode r = nearest_node_g<float>(T.grid, T.stride, T.coord, T.n, T.inv_step,
                                              T.max_nn_dist, T.x0[0] + (double)d[0],
                                              T.x0[1] + (double)d[1], T.x0[2] + (double)d[2],
                                              T.x0[3] + (double)d[3]);
  *flags |= r.flags;
  const float *row = T.grid + (r.node < 0 ? 0 : r.node) * T.stride;
#pragma unroll
  for (int p = 0; p < NP; ++p) out[p] = r.node < 0 ? __int_as_float(0x7fc00000) : __ldg(row + p);
}

constexpr int kWin32 = 4;                       // window nodes per axis (3 cells)
constexpr int kWinNodes32 = kWin32 * kWin32 * kWin32 * kWin32;

// Table value at X0 + d (sd = dsum32(d)): from the shared window `win` when
// the point's cell fits in it (win_lo = box origin), else from the global
// table; nearest row outside the linear region.
__device__ __forceinline__ void interp32(const Rate32 &P, const float d[S], double sd,
                                         const float4 *win, const int *win_lo, float out[NP],
                                         unsigned *flags) {
  const Table32 &T = P.T;
  int ii[S];
  float tt[S];
  if (cell32(T, d, sd, ii, tt)) {
    const int off = win ? window_cell<kWin32>(ii, win_lo) : -1;
    if (off >= 0) {
      constexpr int w3 = 3, w2 = kWin32 * w3, w1 = kWin32 * w2, w0 = kWin32 * w1;
      interp_nodes32(win + off * 3, w0, w1, w2, w3, tt, out);
    } else {
      const int s3 = 3, s2 = T.n * s3, s1 = T.n * s2;
      const int64_t s0 = (int64_t)T.n * s1;
      const float4 *g = reinterpret_cast<const float4 *>(T.grid);
      interp_nodes32(g + ii[0] * s0 + (int64_t)ii[1] * s1 + (int64_t)ii[2] * s2 + ii[3] * s3,
                     (int)s0, s1, s2, s3, tt, out);
    }
    return;
  }
  nearest_row32(T, d, out, flags);
}

// Gradient-energy and elastic parts of mu at one point: off = s' l - kappa lap
// (spv = 0 without elasticity); mu = table value + off.
__device__ __forceinline__ void mu_offset32(const Rate32 &P, const float lap[S], float spv,
                                            float off[S]) {
#pragma unroll
  for (int c = 0; c < S; ++c) off[c] = fmaf(spv, P.lvec[c], -lap[c] * P.kappa[c]);
}

// Row layout of a point's mu/M values: mu (relative to mu(X0)) 0..3, M_Fe 4,
// M_1..4 5..8, the closure X_Fe 9 (FP64 (1 - sum X0) - sum d, rounded).
__device__ __forceinline__ void chem32(const Rate32 &P, const float d[S], const float lap[S],
                                       float spv, const float4 *win, const int *win_lo,
                                       float out[NPM], unsigned *flags) {
  const double sd = dsum32(d);
  float v[NP], off[S];
  interp32(P, d, sd, win, win_lo, v, flags);
  mu_offset32(P, lap, spv, off);
#pragma unroll
  for (int c = 0; c < S; ++c) out[c] = v[c] + off[c];
#pragma unroll
  for (int c = 0; c < NM; ++c) out[S + c] = v[S + c];
  out[NP] = (float)(P.c_fe - sd);
}

// chem32 of two points at once: when both lie in the linear region of one
// table cell, each corner node is loaded once and accumulated into both
// (the same terms in the same order as chem32, so the same bits); otherwise
// each point takes chem32's own path.  hasB = false evaluates A alone.
__device__ __forceinline__ void chem32_pair(const Rate32 &P, const float dA[S], const float lapA[S],
                                            float spA, const float dB[S], const float lapB[S],
                                            float spB, bool hasB, float outA[NPM],
                                            float outB[NPM], unsigned *flags) {
  const Table32 &T = P.T;
  const double sdA = dsum32(dA), sdB = dsum32(dB);
  int iA[S], iB[S];
  float tA[S], tB[S];
  const bool linA = cell32(T, dA, sdA, iA, tA);
  const bool linB = hasB && cell32(T, dB, sdB, iB, tB);
  const bool share = linA && linB && iA[0] == iB[0] && iA[1] == iB[1] && iA[2] == iB[2] &&
                     iA[3] == iB[3];
  float vA[NP], vB[NP];
  if (share) {
    const int s3 = 3, s2 = T.n * s3, s1 = T.n * s2;
    const int64_t s0 = (int64_t)T.n * s1;
    const float4 *base = reinterpret_cast<const float4 *>(T.grid) + iA[0] * s0 +
                         (int64_t)iA[1] * s1 + (int64_t)iA[2] * s2 + iA[3] * s3;
    const Weights32 WA = weights32(tA), WB = weights32(tB);
#pragma unroll
    for (int c = 0; c < 16; ++c) {
      const int b0 = (c >> 3) & 1, b1 = (c >> 2) & 1, b2 = (c >> 1) & 1, b3 = c & 1;
      const float4 *node = base + b0 * s0 + b1 * s1 + b2 * s2 + b3 * s3;
      const float4 a = __ldg(node), b = __ldg(node + 1), e = __ldg(node + 2);
      corner_acc32(c, WA.wa[c >> 2] * WA.wb[c & 3], a, b, e, vA);
      corner_acc32(c, WB.wa[c >> 2] * WB.wb[c & 3], a, b, e, vB);
    }
  } else {
    interp32(P, dA, sdA, nullptr, nullptr, vA, flags);
    if (hasB) interp32(P, dB, sdB, nullptr, nullptr, vB, flags);
  }
  float off[S];
  mu_offset32(P, lapA, spA, off);
#pragma unroll
  for (int c = 0; c < S; ++c) outA[c] = vA[c] + off[c];
#pragma unroll
  for (int c = 0; c < NM; ++c) outA[S + c] = vA[S + c];
  outA[NP] = (float)(P.c_fe - sdA);
  if (hasB) {
    mu_offset32(P, lapB, spB, off);
#pragma unroll
    for (int c = 0; c < S; ++c) outB[c] = vB[c] + off[c];
#pragma unroll
    for (int c = 0; c < NM; ++c) outB[S + c] = vB[S + c];
    outB[NP] = (float)(P.c_fe - sdB);
  }
}

// Face flux (phasefield5d/solver/fluxes.py:128-160) in FP32 between a lower
// position c and an upper position n along one axis, from each position's
// D = X - X0, mu, M_1..4 and (M_Fe, X_Fe):
//   J_a = Xm_a (w_fe <Xm,g> - sum_k Xm_k M_k dk_k) + Xm_a M_a dk_a,
//   dk = g - <Xm,g>, w_fe = X_Fe M_Fe,
// which is the reference's expression regrouped.  The flux is linear in the
// face mobilities and in the mu gradient, so it is evaluated with the sums
// Mc + Mn (for 2 x the mean) and the difference mu_n - mu_c (for dx x the
// gradient): the returned J is (2 dx) times the flux, and kernels scale the
// divergence sum by flux_scale = 0.5 / dx^2.  X_Fe at the face is the mean
// of the two positions' FP64-formed closures.  The units are built without
// multiply-add contraction, so a face gives the same bits whichever of its
// cells (or kernels) evaluates it, and the flux form conserves mass exactly.
__device__ __forceinline__ float4 face_flux32(const Rate32 &P, const float4 &dc, const float4 &muc,
                                              const float4 &mc, const float2 &fc, const float4 &dn,
                                              const float4 &mun, const float4 &mn,
                                              const float2 &fn) {
  const float xm0 = fmaf(0.5f, dc.x + dn.x, P.x0f[0]), xm1 = fmaf(0.5f, dc.y + dn.y, P.x0f[1]),
              xm2 = fmaf(0.5f, dc.z + dn.z, P.x0f[2]), xm3 = fmaf(0.5f, dc.w + dn.w, P.x0f[3]);
  const float g0 = mun.x - muc.x, g1 = mun.y - muc.y, g2 = mun.z - muc.z, g3 = mun.w - muc.w;
  const float w_fe = (0.5f * (fc.y + fn.y)) * (fc.x + fn.x);
  float dot = xm0 * g0;
  dot = fmaf(xm1, g1, dot);
  dot = fmaf(xm2, g2, dot);
  dot = fmaf(xm3, g3, dot);
  const float dk0 = g0 - dot, dk1 = g1 - dot, dk2 = g2 - dot, dk3 = g3 - dot;
  const float w0 = xm0 * (mc.x + mn.x), w1 = xm1 * (mc.y + mn.y), w2 = xm2 * (mc.z + mn.z),
              w3 = xm3 * (mc.w + mn.w);
  float swk = w0 * dk0;
  swk = fmaf(w1, dk1, swk);
  swk = fmaf(w2, dk2, swk);
  swk = fmaf(w3, dk3, swk);
  const float com = fmaf(w_fe, dot, -swk);
  return make_float4(fmaf(w0, dk0, xm0 * com), fmaf(w1, dk1, xm1 * com), fmaf(w2, dk2, xm2 * com),
                     fmaf(w3, dk3, xm3 * com));
}

// Fold this thread's max |dX/dt| into the block and store the block's max
// in `slot` (a plain store: no same-address atomics, no fences); a separate
// one-block kernel reduces the slots and runs the FP64 dt controller.
__device__ __forceinline__ void finish_slot32(float m32, double *red, double *slot) {
  double m = (double)m32;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  const int tid = threadIdx.y * blockDim.x + threadIdx.x;
  const int nw = (blockDim.x * blockDim.y + 31) >> 5;
  __syncthreads();
  if ((tid & 31) == 0) red[tid >> 5] = m;
  __syncthreads();
  if (tid == 0) {
    for (int w = 1; w < nw; ++w) m = fmax(m, red[w]);
    *slot = m;
  }
}

__device__ __forceinline__ void finish_rate32(const Rate32 &P, float m32, double *red) {
  finish_slot32(m32, red, P.partial + (blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x);
}

// The dt controller of one solve from the block maxima slots[0..n): max
// |dX/dt|, the adaptive-dt rule (system.py:90-112), dt / time / step.  Called
// by one warp; lane 0 writes the state.
__device__ __forceinline__ void dt_from_slots32(const Rate32 &P, const double *slots, int n) {
  StepState32 *st = P.st;
  double m = 0.0;
  for (int i = threadIdx.x & 31; i < n; i += 32) m = fmax(m, slots[i]);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) {
    double dt = st->dt;
    if (P.adaptive) dt = adaptive_dt(dt, m, P.ctld, P.t_cfl, P.lower, P.upper, P.factor);
    st->dt = dt;
    st->time = st->time + dt;
    st->xdotmax = m;
    st->step = st->step + 1;
  }
}

// Face flux between two positions of shared-memory SoA planes: D rows at
// XL[c * PX + pl] (lower) and XH[c * PX + ph] (upper), mu/M rows (NPM, in
// chem32's order) at ML[r * PM + ql] and MH[r * PM + qh].
template <int PX, int PM>
__device__ __forceinline__ void face32_between(const Rate32 &P, const float *XL, const float *ML,
                                               int pl, int ql, const float *XH, const float *MH,
                                               int ph, int qh, float J[S]) {
  auto d4 = [](const float *X, int p) {
    return make_float4(X[p], X[PX + p], X[2 * PX + p], X[3 * PX + p]);
  };
  auto mu4 = [](const float *M, int q) {
    return make_float4(M[q], M[PM + q], M[2 * PM + q], M[3 * PM + q]);
  };
  auto m4 = [](const float *M, int q) {
    return make_float4(M[5 * PM + q], M[6 * PM + q], M[7 * PM + q], M[8 * PM + q]);
  };
  auto f2 = [](const float *M, int q) { return make_float2(M[4 * PM + q], M[9 * PM + q]); };
  const float4 j = face_flux32(P, d4(XL, pl), mu4(ML, ql), m4(ML, ql), f2(ML, ql), d4(XH, ph),
                               mu4(MH, qh), m4(MH, qh), f2(MH, qh));
  J[0] = j.x;
  J[1] = j.y;
  J[2] = j.z;
  J[3] = j.w;
}

template <int TX, int TY>
__device__ __forceinline__ void plane_faces32(const Rate32 &P, const float *Xp, const float *Mp,
                                              float *Fx, float *Fy, int tid) {
  using G = PlaneGeom<TX, TY>;
  for (int f = tid; f < G::NFX + G::NFY; f += G::NT) {
    float J[S];
    if (f < G::NFX) {
      const int fy = f / (TX + 1), fx = f - fy * (TX + 1);
      const int pl = (fy + 2) * G::HX + (fx + 1), ql = (fy + 1) * G::MX + fx;
      face32_between<G::PX, G::PM>(P, Xp, Mp, pl, ql, Xp, Mp, pl + 1, ql + 1, J);
#pragma unroll
      for (int c = 0; c < S; ++c) Fx[c * G::NFX + f] = J[c];
    } else {
      const int f2 = f - G::NFX;
      const int fy = f2 / TX, fx = f2 - fy * TX;
      const int pl = (fy + 1) * G::HX + (fx + 2), ql = fy * G::MX + (fx + 1);
      face32_between<G::PX, G::PM>(P, Xp, Mp, pl, ql, Xp, Mp, pl + G::HX, ql + G::MX, J);
#pragma unroll
      for (int c = 0; c < S; ++c) Fy[c * G::NFY + f2] = J[c];
    }
  }
}

template <int TX, int TY>
__device__ __forceinline__ void load_plane32(const float4 *__restrict__ D, int64_t plane_off,
                                             const int *wx, const int *wy, int nx, float *dst,
                                             int tid) {
  using G = PlaneGeom<TX, TY>;
  for (int pos = tid; pos < G::PX; pos += G::NT) {
    const int hy = pos / G::HX, hx = pos - hy * G::HX;
    const float4 v = __ldg(D + plane_off + (int64_t)wy[hy] * nx + wx[hx]);
    dst[0 * G::PX + pos] = v.x;
    dst[1 * G::PX + pos] = v.y;
    dst[2 * G::PX + pos] = v.z;
    dst[3 * G::PX + pos] = v.w;
  }
}

__device__ __forceinline__ void store_rate(float4 *dX, int64_t g, const float out[S], float &vmax) {
#pragma unroll
  for (int c = 0; c < S; ++c) vmax = fmaxf(vmax, fabsf(out[c]));
  dX[g] = make_float4(out[0], out[1], out[2], out[3]);
}


// Skip test for mu/M positions: corners of the halo ring are never used;
// interior_only keeps the tile positions only.
template <int MX, int MY>
__device__ __forceinline__ bool skip_pos(int mx, int my, bool interior_only) {
  const bool ex = (mx == 0 || mx == MX - 1), ey = (my == 0 || my == MY - 1);
  return interior_only ? (ex || ey) : (ex && ey);
}

// Shared-memory scratch of a per-tile cell sort: hist[256], wsum[NT/32+1],
// order/rank/key per mu/M position.
struct SortScratch32 {
  int *hist;
  int *wsum;
  unsigned short *order;
  unsigned short *rank;
  unsigned char *key;
};

template <int TX, int TY>
struct SortBytes32 {
  using G = PlaneGeom<TX, TY>;
  static constexpr size_t bytes = (256 + G::NT / 32 + 1) * sizeof(int) + G::PM * (2 * 2 + 1);
  static __device__ __forceinline__ SortScratch32 carve(void *base) {
    SortScratch32 s;
    s.hist = reinterpret_cast<int *>(base);
    s.wsum = s.hist + 256;
    s.order = reinterpret_cast<unsigned short *>(s.wsum + G::NT / 32 + 1);
    s.rank = s.order + G::PM;
    s.key = reinterpret_cast<unsigned char *>(s.rank + G::PM);
    return s;
  }
};

// mu/M of one plane (tile + 1-cell halo, or the tile only) into dst.  Xm/Xp
// are the neighbouring planes along axis 0 in 3D (nullptr in 2D, where the
// y-neighbours sit in the same plane).  Stages the table window first.
// SORT: positions evaluated in table-cell order (cell_hash counting sort),
// so the lanes of a warp gather the same table nodes; only the thread that
// evaluates a position changes.  SORT = 2: a thread evaluates two
// consecutive positions of that order with chem32_pair, which shares the
// corner loads when they lie in one table cell (no table window).
template <int TX, int TY, int DIM, bool WIN, int SORT = 0>
__device__ __forceinline__ void mu_plane32(const Rate32 &P, const float *Xm, const float *Xc,
                                           const float *Xp, float *dst, int64_t zoff,
                                           const int *wx, const int *wy, bool interior_only,
                                           float4 *win, int *red, int *win_lo, unsigned *flags,
                                           int tid, SortScratch32 ss = {}) {
  using G = PlaneGeom<TX, TY>;
  // 1. table window around the tile centre's cell (reloaded if it moved).
  int rep[S];
  float tr[S];
  float dc[S];
  const int cp = (TY / 2 + 2) * G::HX + (TX / 2 + 2);
#pragma unroll
  for (int c = 0; c < S; ++c) dc[c] = Xc[c * G::PX + cp];
  const bool use_win = WIN && cell32(P.T, dc, dsum32(dc), rep, tr);
  int o[S] = {0, 0, 0, 0};
  if (use_win) {
    window_origin<kWin32>(rep, tr, o);
    ensure_window<kWin32, 3, float4, G::NT>(reinterpret_cast<const float4 *>(P.T.grid), P.T.n, o,
                                            win, win_lo, tid);
  }
  // 2. (SORT) table-cell order of the positions.
  int nwork = G::PM;
  if constexpr (SORT) {
    for (int i = tid; i < 256; i += G::NT) ss.hist[i] = 0;
    __syncthreads();
    for (int pos = tid; pos < G::PM; pos += G::NT) {
      const int my = pos / G::MX, mx = pos - my * G::MX;
      if (skip_pos<G::MX, G::MY>(mx, my, interior_only)) {
        ss.rank[pos] = 0xFFFFu;
        continue;
      }
      const int px = (my + 1) * G::HX + (mx + 1);
      float u[S];
#pragma unroll
      for (int c = 0; c < S; ++c)
        u[c] = fmaf(Xc[c * G::PX + px], P.T.inv_step_f, P.T.fb[c]) + (float)P.T.ib[c];
      const int k = cell_hash_u(u);
      ss.key[pos] = (unsigned char)k;
      ss.rank[pos] = (unsigned short)atomicAdd(&ss.hist[k], 1);
    }
    __syncthreads();
    nwork = block_exclusive_scan<256, G::NT>(ss.hist, ss.wsum, tid);
    for (int pos = tid; pos < G::PM; pos += G::NT)
      if (ss.rank[pos] != 0xFFFFu) ss.order[ss.hist[ss.key[pos]] + ss.rank[pos]] = (unsigned short)pos;
    __syncthreads();
  }
  // 3. interpolation + Laplacian + mu assembly.
  auto inputs = [&](int pos, float d[S], float lap[S], float &spv) {
    const int my = pos / G::MX, mx = pos - my * G::MX;
    const int px = (my + 1) * G::HX + (mx + 1);
#pragma unroll
    for (int c = 0; c < S; ++c) {
      const float *q = Xc + c * G::PX;
      d[c] = q[px];
      if (DIM == 3) {
        const float nb[6] = {Xp[c * G::PX + px], Xm[c * G::PX + px], q[px + G::HX], q[px - G::HX],
                             q[px + 1], q[px - 1]};
        lap[c] = lap32<6>(nb, d[c], P.inv_dx2);
      } else {
        const float nb[4] = {q[px + G::HX], q[px - G::HX], q[px + 1], q[px - 1]};
        lap[c] = lap32<4>(nb, d[c], P.inv_dx2);
      }
    }
    spv = P.sp ? __ldg(P.sp + zoff + (int64_t)wy[my + 1] * P.nx + wx[mx + 1]) : 0.f;
  };
  if constexpr (SORT == 2) {
    for (int w = 2 * tid; w < nwork; w += 2 * G::NT) {
      const int posA = ss.order[w];
      const bool hasB = w + 1 < nwork;
      const int posB = hasB ? (int)ss.order[w + 1] : posA;
      float dA[S], lapA[S], dB[S], lapB[S], spA, spB, vA[NPM], vB[NPM];
      inputs(posA, dA, lapA, spA);
      inputs(posB, dB, lapB, spB);
      chem32_pair(P, dA, lapA, spA, dB, lapB, spB, hasB, vA, vB, flags);
#pragma unroll
      for (int r = 0; r < NPM; ++r) dst[r * G::PM + posA] = vA[r];
      if (hasB) {
#pragma unroll
        for (int r = 0; r < NPM; ++r) dst[r * G::PM + posB] = vB[r];
      }
    }
  } else {
  for (int w = tid; w < nwork; w += G::NT) {
    const int pos = SORT ? (int)ss.order[w] : w;
    const int my = pos / G::MX, mx = pos - my * G::MX;
    if (!SORT && skip_pos<G::MX, G::MY>(mx, my, interior_only)) continue;
    const int px = (my + 1) * G::HX + (mx + 1);
    float d[S], lap[S];
#pragma unroll
    for (int c = 0; c < S; ++c) {
      const float *q = Xc + c * G::PX;
      d[c] = q[px];
      if (DIM == 3) {
        const float nb[6] = {Xp[c * G::PX + px], Xm[c * G::PX + px], q[px + G::HX], q[px - G::HX],
                             q[px + 1], q[px - 1]};
        lap[c] = lap32<6>(nb, d[c], P.inv_dx2);
      } else {
        const float nb[4] = {q[px + G::HX], q[px - G::HX], q[px + 1], q[px - 1]};
        lap[c] = lap32<4>(nb, d[c], P.inv_dx2);
      }
    }
    const float spv = P.sp ? __ldg(P.sp + zoff + (int64_t)wy[my + 1] * P.nx + wx[mx + 1]) : 0.f;
    float v[NPM];
    chem32(P, d, lap, spv, use_win ? win : nullptr, o, v, flags);
#pragma unroll
    for (int r = 0; r < NPM; ++r) dst[r * G::PM + pos] = v[r];
  }
  }
}

// mu/M of one plane (tile + 1-cell halo, or the tile only) read from the
// split buffers (written by k32_chem) into dst, in mu_plane32's layout.
template <int TX, int TY>
__device__ __forceinline__ void load_mu_plane32(const Rate32 &P, int64_t zoff, const int *wx,
                                                const int *wy, bool interior_only, float *dst,
                                                int tid) {
  using G = PlaneGeom<TX, TY>;
  for (int pos = tid; pos < G::PM; pos += G::NT) {
    const int my = pos / G::MX, mx = pos - my * G::MX;
    if (skip_pos<G::MX, G::MY>(mx, my, interior_only)) continue;
    const int64_t g = zoff + (int64_t)wy[my + 1] * P.nx + wx[mx + 1];
    const float4 mu = __ldg(P.mm_mu + g), m = __ldg(P.mm_m + g);
    const float2 f = __ldg(P.mm_f + g);
    const float v[NPM] = {mu.x, mu.y, mu.z, mu.w, f.x, m.x, m.y, m.z, m.w, f.y};
#pragma unroll
    for (int r = 0; r < NPM; ++r) dst[r * G::PM + pos] = v[r];
  }
}

// Shared memory common to the plane kernels, after the kernel-specific
// arrays: block-max scratch (double), the table window (float4), window
// reduction scratch and origin (int), halo index tables (int).
template <int TX, int TY>
struct Smem32Tail {
  using G = PlaneGeom<TX, TY>;
  static constexpr size_t bytes = (G::NT / 32) * sizeof(double) + kWinNodes32 * 3 * sizeof(float4) +
                                  (S * (G::NT / 32) + S + 1) * sizeof(int) +
                                  (G::HX + G::HY) * sizeof(int);
};


// (h, l) += inc with TwoSum and renormalisation; explicit _rn intrinsics keep
// every operation separately rounded.
__device__ __forceinline__ void comp_add(float &h, float &l, float inc) {
  const float s = __fadd_rn(h, inc);
  const float bb = __fsub_rn(s, h);
  const float err = __fadd_rn(__fsub_rn(h, __fsub_rn(s, bb)), __fsub_rn(inc, bb));
  const float lo = __fadd_rn(l, err);
  const float hn = __fadd_rn(s, lo);
  l = __fsub_rn(lo, __fsub_rn(hn, s));
  h = hn;
}

__device__ __forceinline__ unsigned oob_flags_x(const double x[S]) {
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

__device__ __forceinline__ void raise32(StepState32 *st, unsigned f) {
  if (!f) return;
  atomicOr(&st->flags, f);
  if (f & (PF5D_FLAG_NONFINITE | PF5D_FLAG_OOB_HARD)) atomicExch(&st->halt, 1u);
}


// ------------------------------------------------------------------------
// One 2D plane tile of a solve (shared by the single-solve and batched
// kernels).  Shared-memory layout, in order: table window, block-max
// scratch, X (tile + 2 halo), mu/M (tile + 1 halo), x- and y-face fluxes,
// window scratch/origin, halo index tables.
// ------------------------------------------------------------------------
template <int TX, int TY, int SORT = 0>
struct Tile2dSmem32 {
  using G = PlaneGeom<TX, TY>;
  static constexpr size_t bytes = Smem32Tail<TX, TY>::bytes +
      (S * G::PX + NPM * G::PM + S * G::NFX + S * G::NFY) * sizeof(float) +
      (SORT ? SortBytes32<TX, TY>::bytes : 0);
  static __device__ __forceinline__ double *red(float4 *sm4) {
    return reinterpret_cast<double *>(sm4 + kWinNodes32 * 3);
  }
};

// Evaluates tile (bx, by) of solve P and writes its dX/dt; returns this
// thread's max |dX/dt|.  Ends with all threads past a barrier.
template <int TX, int TY, bool WIN, int SORT = 0, bool SPLIT = false, bool PERPOINT = false>
__device__ __forceinline__ float tile2d32_body(const Rate32 &P, int bx, int by, float4 *sm4,
                                               unsigned *flags, int tid) {
  using G = PlaneGeom<TX, TY>;
  float4 *win = sm4;
  double *red = Tile2dSmem32<TX, TY>::red(sm4);
  float *Xs = reinterpret_cast<float *>(red + G::NT / 32);
  float *Ms = Xs + S * G::PX;
  float *Fx = Ms + NPM * G::PM;
  float *Fy = Fx + S * G::NFX;
  int *wred = reinterpret_cast<int *>(Fy + S * G::NFY);
  int *win_lo = wred + S * (G::NT / 32);
  int *wx = win_lo + S + 1;
  int *wy = wx + G::HX;
  SortScratch32 ss{};
  if constexpr (SORT) ss = SortBytes32<TX, TY>::carve(wy + G::HY);
  const int tx = tid % TX, ty = tid / TX;
  const int x0 = bx * TX, y0 = by * TY;
  if (tid == 0) win_lo[S] = 0;
  for (int i = tid; i < G::HX + G::HY; i += G::NT) {
    if (i < G::HX) wx[i] = wrap_any(x0 + i - 2, P.nx);
    else wy[i - G::HX] = wrap_any(y0 + (i - G::HX) - 2, P.ny);
  }
  __syncthreads();
  load_plane32<TX, TY>(P.D, 0, wx, wy, P.nx, Xs, tid);
  __syncthreads();
  if constexpr (SPLIT)
    load_mu_plane32<TX, TY>(P, 0, wx, wy, false, Ms, tid);
  else
    mu_plane32<TX, TY, 2, WIN, SORT>(P, nullptr, Xs, nullptr, Ms, 0, wx, wy, false, win, wred,
                                     win_lo, flags, tid, ss);
  __syncthreads();
  float vmax = 0.f;
  if constexpr (PERPOINT) {
    // each point evaluates its four faces (each face is evaluated by both of
    // its cells, with identical operands and operation order)
    if (x0 + tx < P.nx && y0 + ty < P.ny) {
      const int pX = (ty + 2) * G::HX + (tx + 2), pM = (ty + 1) * G::MX + (tx + 1);
      float jyp[S], jym[S], jxp[S], jxm[S], out[S];
      face32_between<G::PX, G::PM>(P, Xs, Ms, pX, pM, Xs, Ms, pX + G::HX, pM + G::MX, jyp);
      face32_between<G::PX, G::PM>(P, Xs, Ms, pX - G::HX, pM - G::MX, Xs, Ms, pX, pM, jym);
      face32_between<G::PX, G::PM>(P, Xs, Ms, pX, pM, Xs, Ms, pX + 1, pM + 1, jxp);
      face32_between<G::PX, G::PM>(P, Xs, Ms, pX - 1, pM - 1, Xs, Ms, pX, pM, jxm);
#pragma unroll
      for (int c = 0; c < S; ++c)
        out[c] = __fmul_rn(__fadd_rn(__fsub_rn(jyp[c], jym[c]), __fsub_rn(jxp[c], jxm[c])),
                           P.flux_scale);
      store_rate(P.dX, (int64_t)(y0 + ty) * P.nx + (x0 + tx), out, vmax);
    }
    return vmax;                     // (shared memory still being read: callers sync first)
  }
  plane_faces32<TX, TY>(P, Xs, Ms, Fx, Fy, tid);
  __syncthreads();
  if (x0 + tx < P.nx && y0 + ty < P.ny) {
    float out[S];
#pragma unroll
    for (int c = 0; c < S; ++c) {
      const float ay = __fsub_rn(Fy[c * G::NFY + (ty + 1) * TX + tx], Fy[c * G::NFY + ty * TX + tx]);
      const float ax = __fsub_rn(Fx[c * G::NFX + ty * (TX + 1) + tx + 1], Fx[c * G::NFX + ty * (TX + 1) + tx]);
      out[c] = __fmul_rn(__fadd_rn(ay, ax), P.flux_scale);
    }
    store_rate(P.dX, (int64_t)(y0 + ty) * P.nx + (x0 + tx), out, vmax);
  }
  return vmax;
}

}  // namespace pf5d
