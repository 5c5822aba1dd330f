// pf5d_window.cuh -- shared-memory table window for the fused rate kernels.
//
// The points of one plane tile fall into a handful of table cells (their
// compositions differ by a fraction of a cell), so the block stages a
// W x W x W x W box of table nodes in shared memory and the 16-corner
// interpolation reads it there instead of issuing 16 scattered global
// gathers per point.  The box is placed around the cell of the tile's
// centre point (every thread derives the same origin from the same staged
// value, so no reduction is needed) and is reloaded only when that origin
// moves; points whose cell does not fit in the box read the global table as
// before, so the result never depends on the box.
#pragma once


#include "pf5d_device.cuh"

namespace pf5d {

// Copy the W^4 node box starting at node `lo` (shared) from the global
// table into `win`: node (a,b,c,d) of the box at ((a*W+b)*W+c)*W+d, each
// node NV vectors of type V.  Nodes beyond the table edge are left unset
// (no cell can reference them: cells use nodes i..i+1 with i <= n-2).
template <int W, int NV, typename V, int NT>
__device__ __forceinline__ void load_window(const V *__restrict__ grid_v, int n, const int *lo,
                                            V *win, int tid) {
  constexpr int NODES = W * W * W * W;
  for (int q = tid; q < NODES * NV; q += NT) {
    const int node = q / NV, part = q - node * NV;
    const int a = node / (W * W * W), b = (node / (W * W)) % W, c = (node / W) % W, d = node % W;
    const int g0 = lo[0] + a, g1 = lo[1] + b, g2 = lo[2] + c, g3 = lo[3] + d;
    if (g0 < n && g1 < n && g2 < n && g3 < n) {
      const int64_t gn = (((int64_t)g0 * n + g1) * n + g2) * n + g3;
      win[q] = __ldg(grid_v + gn * NV + part);
    }
  }
}

// Offset (in nodes) of cell `cell` inside the box, or -1 if it does not fit.
template <int W>
__device__ __forceinline__ int window_cell(const int cell[S], const int *lo) {
  int off = 0;
#pragma unroll
  for (int a = 0; a < S; ++a) {
    const int r = cell[a] - lo[a];
    if (r < 0 || r > W - 2) return -1;
    off = off * W + r;
  }
  return off;
}

// Box origin for a representative point in cell `rep` with fractional
// coordinates `t`: one node below the node nearest to it, so the box spans
// the cells on both sides of that node (W = 3) and one more above (W = 4).
// Compositions near a table node straddle two cells; anchoring on the
// nearest node keeps the origin fixed while they do.
template <int W, typename R>
__device__ __forceinline__ void window_origin(const int rep[S], const R t[S], int o[S]) {
#pragma unroll
  for (int a = 0; a < S; ++a) {
    const int v = rep[a] + (t[a] < R(0.5) ? 0 : 1) - 1;
    o[a] = v < 0 ? 0 : v;
  }
}

// Make `win` hold the box at origin o (shared win_lo[0..3] and win_lo[4] =
// valid flag track what is loaded).  Uniform: every thread passes the same o.
template <int W, int NV, typename V, int NT>
__device__ __forceinline__ void ensure_window(const V *__restrict__ grid_v, int n, const int o[S],
                                              V *win, int *win_lo, int tid) {
  const bool same = win_lo[4] && win_lo[0] == o[0] && win_lo[1] == o[1] && win_lo[2] == o[2] &&
                    win_lo[3] == o[3];
  if (same) return;
  __syncthreads();                   // every thread has read win_lo and left the old box
  if (tid < S) win_lo[tid] = o[tid];
  if (tid == 0) win_lo[4] = 1;
  load_window<W, NV, V, NT>(grid_v, n, o, win, tid);
  __syncthreads();
}

}  // namespace pf5d
