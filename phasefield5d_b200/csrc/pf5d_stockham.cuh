// pf5d_stockham.cuh -- in-shared-memory complex FFTs of a power-of-two
// length for the elastic-term kernels (the column pass and the fused
// update + row transform): mixed-radix Stockham autosort, radix-8 stages
// then one radix-4 or radix-2 stage, natural order after every stage;
// forward exp(-2 pi i jk/N), inverse exp(+2 pi i jk/N), both unnormalised.
// A block of kColThreads threads transforms one sequence of N complex
// values in shared memory (x and y ping-pong; the result pointer is
// returned).
#pragma once

#include <cuda_runtime.h>

namespace pf5d {

constexpr int kColThreads = 256;

// complex type traits of the column pass (FP64 double2, FP32c float2)
template <typename C> struct CT;
template <> struct CT<double2> { using R = double; };
template <> struct CT<float2> { using R = float; };
template <typename C>
__device__ __forceinline__ C cmk(typename CT<C>::R a, typename CT<C>::R b) {
  C c;
  c.x = a;
  c.y = b;
  return c;
}

template <typename C>
__device__ __forceinline__ C cmul(C a, C b) {
  return cmk<C>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
template <typename C>
__device__ __forceinline__ C cadd(C a, C b) { return cmk<C>(a.x + b.x, a.y + b.y); }
template <typename C>
__device__ __forceinline__ C csub(C a, C b) { return cmk<C>(a.x - b.x, a.y - b.y); }
// times -i (forward) or +i (inverse)
template <typename C, bool INV>
__device__ __forceinline__ C crot(C a) {
  return INV ? cmk<C>(-a.y, a.x) : cmk<C>(a.y, -a.x);
}

template <typename C, bool INV>
__device__ __forceinline__ void dft4(C *u) {
  const C c0 = cadd(u[0], u[2]), c1 = cadd(u[1], u[3]);
  const C d0 = csub(u[0], u[2]), d1 = crot<C, INV>(csub(u[1], u[3]));
  u[0] = cadd(c0, c1);
  u[1] = cadd(d0, d1);
  u[2] = csub(c0, c1);
  u[3] = csub(d0, d1);
}

// Radix-8 by decimation in frequency: two length-4 transforms of the sums
// and of the twiddled differences (W8^n, n < 4).
template <typename C, bool INV>
__device__ __forceinline__ void dft8(C *v) {
  constexpr typename CT<C>::R h = (typename CT<C>::R)0.70710678118654752440;
  C a[4], b[4];
#pragma unroll
  for (int n = 0; n < 4; ++n) {
    a[n] = cadd(v[n], v[n + 4]);
    b[n] = csub(v[n], v[n + 4]);
  }
  b[1] = cmul(b[1], cmk<C>(h, INV ? h : -h));
  b[2] = crot<C, INV>(b[2]);
  b[3] = cmul(b[3], cmk<C>(-h, INV ? h : -h));
  dft4<C, INV>(a);
  dft4<C, INV>(b);
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    v[2 * k] = a[k];
    v[2 * k + 1] = b[k];
  }
}

template <typename C, int R, bool INV>
__device__ __forceinline__ void dftr(C *v) {
  if constexpr (R == 8) {
    dft8<C, INV>(v);
  } else if constexpr (R == 4) {
    dft4<C, INV>(v);
  } else {
    const C a = v[0];
    v[0] = cadd(a, v[1]);
    v[1] = csub(a, v[1]);
  }
}

// One Stockham stage of radix R over span ns, x -> y, then a barrier.
// tw[t] = exp(-2 pi i t / N0), t < N0.
template <typename C, int N0, int R, bool INV>
__device__ __forceinline__ void stockham_stage(const C *x, C *y,
                                               const C *__restrict__ tw, int ns, int tid) {
  constexpr int Q = N0 / R;
  for (int j = tid; j < Q; j += kColThreads) {
    const C *xc = x;
    C *yc = y;
    const int m = j & (ns - 1);
    const int step = m * (N0 / (R * ns));
    C v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      v[r] = xc[j + r * Q];
      if (r > 0) {
        C w = tw[r * step];
        if (INV) w.y = -w.y;
        v[r] = cmul(v[r], w);
      }
    }
    dftr<C, R, INV>(v);
    const int d = (j - m) * R + m;
#pragma unroll
    for (int r = 0; r < R; ++r) yc[d + r * ns] = v[r];
  }
  __syncthreads();
}

template <typename C, int N0, bool INV>
__device__ __forceinline__ C *stockham(C *x, C *y, const C *__restrict__ tw,
                                             int tid) {
  int ns = 1;
#pragma unroll 1
  for (; ns * 8 <= N0; ns *= 8) {
    stockham_stage<C, N0, 8, INV>(x, y, tw, ns, tid);
    C *t = x;
    x = y;
    y = t;
  }
  if (ns < N0) {
    if (N0 / ns >= 4) stockham_stage<C, N0, 4, INV>(x, y, tw, ns, tid);
    else stockham_stage<C, N0, 2, INV>(x, y, tw, ns, tid);
    C *t = x;
    x = y;
    y = t;
  }
  return x;
}


}  // namespace pf5d
