/*
 * pf5d_oracle.c -- CPU oracle for the phasefield5d Cahn-Hilliard step loop.
 *
 * TEST INFRASTRUCTURE ONLY.  This file restates, in plain C, the reference's
 * per-step kernels so tests, the smoke check and the CPU-baseline leg of the
 * benchmark have a checker.  Nothing in the product imports, links or runs
 * it; the product path is the CUDA library under phasefield5d_b200/csrc.
 *
 * Every routine keeps the reference's floating-point operation order and is
 * compiled with -ffp-contract=off (no FMA), which is what Numba's
 * fastmath=False code does, so results are bit-identical to the reference's
 * Numba kernels.  Each routine cites the reference function it restates
 * (paths relative to the phasefield5d project root).
 *
 * Arrays follow the reference layout: C-contiguous (*spatial, S) float64,
 * S = number of independent components.  Views such as mu = interp[..., :4]
 * and M = interp[..., 4:] are passed as (pointer, point stride).
 */
#include <math.h>
#include <stdint.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define PF5D_ORACLE_API __attribute__((visibility("default")))

static inline int64_t wrap_p(int64_t i, int64_t n) { return i + 1 < n ? i + 1 : 0; }
static inline int64_t wrap_m(int64_t i, int64_t n) { return i - 1 >= 0 ? i - 1 : n - 1; }

/* --------------------------------------------------------------------------
 * Interpolation (phasefield5d/solver/interpolation.py:67-147)
 * ------------------------------------------------------------------------ */

/* mask[i] = (sum_d comp[i,d] <= threshold), summed left to right from 0.0
 * (interpolation.py:67-79). */
PF5D_ORACLE_API void orc_linear_mask(const double *comp, int64_t npts, int S,
                                     double threshold, uint8_t *mask) {
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < npts; ++i) {
    double s = 0.0;
    for (int d = 0; d < S; ++d) s += comp[i * S + d];
    mask[i] = (s <= threshold);
  }
}

static inline void axis_coord(double u, int num, int *i, double *t) {
  /* interpolation.py:110-121 */
  if (u <= 0.0) { *i = 0; *t = 0.0; }
  else if (u >= (double)(num - 1)) { *i = num - 2; *t = 1.0; }
  else { *i = (int)u; *t = u - (double)(*i); }
}

/* Quadrilinear interpolation of all props; masked-out rows get NaN
 * (interpolation.py:86-147).  16 weights as ((a*b)*c)*d products in the listed
 * corner order; per prop, the 16 terms are summed left to right. */
PF5D_ORACLE_API void orc_interp4d(const double *comp, int64_t npts, const double *grid,
                                  int num, int nprops, double step, double *out,
                                  const uint8_t *mask) {
  const double inv_step = 1.0 / step;
  const int64_t s3 = nprops, s2 = (int64_t)num * s3, s1 = (int64_t)num * s2,
                s0 = (int64_t)num * s1;
#pragma omp parallel for schedule(static)
  for (int64_t idx = 0; idx < npts; ++idx) {
    double *o = out + idx * nprops;
    if (!mask[idx]) {
      for (int p = 0; p < nprops; ++p) o[p] = NAN;
      continue;
    }
    int i0, i1, i2, i3;
    double t0, t1, t2, t3;
    axis_coord(comp[idx * 4 + 0] * inv_step, num, &i0, &t0);
    axis_coord(comp[idx * 4 + 1] * inv_step, num, &i1, &t1);
    axis_coord(comp[idx * 4 + 2] * inv_step, num, &i2, &t2);
    axis_coord(comp[idx * 4 + 3] * inv_step, num, &i3, &t3);
    const double q0 = 1.0 - t0, q1 = 1.0 - t1, q2 = 1.0 - t2, q3 = 1.0 - t3;
    double w[16];
    w[0] = q0 * q1 * q2 * q3;  w[1] = q0 * q1 * q2 * t3;
    w[2] = q0 * q1 * t2 * q3;  w[3] = q0 * q1 * t2 * t3;
    w[4] = q0 * t1 * q2 * q3;  w[5] = q0 * t1 * q2 * t3;
    w[6] = q0 * t1 * t2 * q3;  w[7] = q0 * t1 * t2 * t3;
    w[8] = t0 * q1 * q2 * q3;  w[9] = t0 * q1 * q2 * t3;
    w[10] = t0 * q1 * t2 * q3; w[11] = t0 * q1 * t2 * t3;
    w[12] = t0 * t1 * q2 * q3; w[13] = t0 * t1 * q2 * t3;
    w[14] = t0 * t1 * t2 * q3; w[15] = t0 * t1 * t2 * t3;
    const double *base = grid + i0 * s0 + i1 * s1 + i2 * s2 + i3 * s3;
    for (int p = 0; p < nprops; ++p) {
      double acc = 0.0;
      for (int c = 0; c < 16; ++c) {
        const int b0 = (c >> 3) & 1, b1 = (c >> 2) & 1, b2 = (c >> 1) & 1, b3 = c & 1;
        const double term = w[c] * base[b0 * s0 + b1 * s1 + b2 * s2 + b3 * s3 + p];
        acc = (c == 0) ? term : acc + term;
      }
      o[p] = acc;
    }
  }
}

/* --------------------------------------------------------------------------
 * Laplacian (phasefield5d/solver/operators.py:32-76)
 * ------------------------------------------------------------------------ */

PF5D_ORACLE_API void orc_laplacian(int dim, const int64_t *shape, int S, const double *c,
                                   double dx, double *out) {
  const double inv_dx2 = 1.0 / (dx * dx);
  if (dim == 1) {
    const int64_t nx = shape[0];
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < nx; ++i) {
      const int64_t ip = wrap_p(i, nx), im = wrap_m(i, nx);
      for (int s = 0; s < S; ++s)
        out[i * S + s] = (c[ip * S + s] + c[im * S + s] - 2.0 * c[i * S + s]) * inv_dx2;
    }
  } else if (dim == 2) {
    const int64_t nx = shape[0], ny = shape[1];
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < nx; ++i) {
      const int64_t ip = wrap_p(i, nx), im = wrap_m(i, nx);
      for (int64_t j = 0; j < ny; ++j) {
        const int64_t jp = wrap_p(j, ny), jm = wrap_m(j, ny);
#define C2(a, b, s) c[((a) * ny + (b)) * S + (s)]
        for (int s = 0; s < S; ++s)
          out[(i * ny + j) * S + s] =
              (C2(ip, j, s) + C2(im, j, s) + C2(i, jp, s) + C2(i, jm, s) - 4.0 * C2(i, j, s)) *
              inv_dx2;
#undef C2
      }
    }
  } else {
    const int64_t nx = shape[0], ny = shape[1], nz = shape[2];
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < nx; ++i) {
      const int64_t ip = wrap_p(i, nx), im = wrap_m(i, nx);
      for (int64_t j = 0; j < ny; ++j) {
        const int64_t jp = wrap_p(j, ny), jm = wrap_m(j, ny);
        for (int64_t k = 0; k < nz; ++k) {
          const int64_t kp = wrap_p(k, nz), km = wrap_m(k, nz);
#define C3(a, b, d, s) c[(((a) * ny + (b)) * nz + (d)) * S + (s)]
          for (int s = 0; s < S; ++s)
            out[((i * ny + j) * nz + k) * S + s] =
                (C3(ip, j, k, s) + C3(im, j, k, s) + C3(i, jp, k, s) + C3(i, jm, k, s) +
                 C3(i, j, kp, s) + C3(i, j, km, s) - 6.0 * C3(i, j, k, s)) *
                inv_dx2;
#undef C3
        }
      }
    }
  }
}

/* mu[p, s] -= lap[p, s] * kappa[s]: the two numpy statements of
 * examples/simulate.py:254-255, one rounding each. */
PF5D_ORACLE_API void orc_kappa_subtract(double *mu, int64_t mu_stride, double *lap,
                                        const double *kappa, int64_t npts, int S) {
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < npts; ++i)
    for (int s = 0; s < S; ++s) {
      lap[i * S + s] = lap[i * S + s] * kappa[s];
      mu[i * mu_stride + s] = mu[i * mu_stride + s] - lap[i * S + s];
    }
}

/* --------------------------------------------------------------------------
 * Elastic helpers (phasefield5d/solver/elastic.py:21-29, 258-263)
 * ------------------------------------------------------------------------ */

/* out[i] = sum_s (X[i,s] - X0[s]) * l[s], accumulated from 0.0. */
PF5D_ORACLE_API void orc_dot_misfit(const double *X, int64_t npts, int S, const double *X0,
                                    const double *l, double *out) {
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < npts; ++i) {
    double acc = 0.0;
    for (int s = 0; s < S; ++s) acc += (X[i * S + s] - X0[s]) * l[s];
    out[i] = acc;
  }
}

/* mu[i, s] += sr[i] * l[s]  (np.multiply into mu_elastic, then +=). */
PF5D_ORACLE_API void orc_expand_add(double *mu, int64_t mu_stride, const double *sr,
                                    const double *l, int64_t npts, int S) {
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < npts; ++i)
    for (int s = 0; s < S; ++s) mu[i * mu_stride + s] = mu[i * mu_stride + s] + sr[i] * l[s];
}

/* --------------------------------------------------------------------------
 * Face flux and fused divergence (phasefield5d/solver/fluxes.py:128-160, 296-395)
 * ------------------------------------------------------------------------ */

/* _face_flux: midpoint composition/mobility, dyadic mobility; S <= 8. */
static inline void face_flux(int S, const double *Xc, const double *Mc, const double *Xn,
                             const double *Mn, const double *g, double *out) {
  double xm[8], mm[9], dk[8];
  for (int a = 0; a < S; ++a) xm[a] = 0.5 * (Xc[a] + Xn[a]);
  for (int a = 0; a <= S; ++a) mm[a] = 0.5 * (Mc[a] + Mn[a]);
  double sum_x = 0.0;
  for (int a = 0; a < S; ++a) sum_x += xm[a];
  const double x_fe = 1.0 - sum_x;
  const double w_fe = x_fe * mm[0];
  double dot_xg = 0.0;
  for (int b = 0; b < S; ++b) dot_xg += xm[b] * g[b];
  const double dot_fe = -dot_xg;
  for (int k = 0; k < S; ++k) dk[k] = g[k] - dot_xg;
  double sum_wk = 0.0;
  for (int k = 0; k < S; ++k) sum_wk += xm[k] * mm[1 + k] * dk[k];
  for (int a = 0; a < S; ++a) {
    const double wa = xm[a] * mm[1 + a];
    out[a] = w_fe * (-xm[a]) * dot_fe + wa * dk[a] - xm[a] * sum_wk;
  }
}

/* dX/dt = div(M grad mu): per cell, forward/backward mu gradients inline, one
 * face flux per face, divergence (fx_p - fx_m + fy_p - fy_m + fz_p - fz_m)*inv_dx
 * left to right. X is (*sp, S) contiguous; M, mu are views with point strides. */
PF5D_ORACLE_API void orc_divergence_from_mu(int dim, const int64_t *shape, int S,
                                            const double *X, const double *M,
                                            int64_t m_stride, const double *mu,
                                            int64_t mu_stride, double inv_dx, double *out) {
  int64_t nx = shape[0], ny = dim > 1 ? shape[1] : 1, nz = dim > 2 ? shape[2] : 1;
  const int64_t npts = nx * ny * nz;
#pragma omp parallel for schedule(static)
  for (int64_t p = 0; p < npts; ++p) {
    const int64_t k = p % nz, j = (p / nz) % ny, i = p / (nz * ny);
    int64_t nb[6];
    int nf = 0;
    /* neighbour point indices in the reference's face order: +x, -x, +y, -y, +z, -z */
    nb[nf++] = (wrap_p(i, nx) * ny + j) * nz + k;
    nb[nf++] = (wrap_m(i, nx) * ny + j) * nz + k;
    if (dim > 1) {
      nb[nf++] = (i * ny + wrap_p(j, ny)) * nz + k;
      nb[nf++] = (i * ny + wrap_m(j, ny)) * nz + k;
    }
    if (dim > 2) {
      nb[nf++] = (i * ny + j) * nz + wrap_p(k, nz);
      nb[nf++] = (i * ny + j) * nz + wrap_m(k, nz);
    }
    double f[6][8];
    for (int fi = 0; fi < nf; ++fi) {
      double g[8];
      const int64_t q = nb[fi];
      for (int s = 0; s < S; ++s)
        g[s] = (fi & 1) ? (mu[p * mu_stride + s] - mu[q * mu_stride + s]) * inv_dx
                        : (mu[q * mu_stride + s] - mu[p * mu_stride + s]) * inv_dx;
      face_flux(S, X + p * S, M + p * m_stride, X + q * S, M + q * m_stride, g, f[fi]);
    }
    for (int s = 0; s < S; ++s) {
      double acc = f[0][s] - f[1][s];
      for (int fi = 2; fi < nf; fi += 2) acc = acc + f[fi][s] - f[fi + 1][s];
      out[p * S + s] = acc * inv_dx;
    }
  }
}

/* Forward/backward gradients along each axis, (dim, *sp, S) outputs
 * (phasefield5d/solver/operators.py:88-123, 126-158, 289-317). */
PF5D_ORACLE_API void orc_gradients_pm(int dim, const int64_t *shape, int S, const double *c,
                                      int64_t c_stride, double dx, double *gp, double *gm) {
  int64_t nx = shape[0], ny = dim > 1 ? shape[1] : 1, nz = dim > 2 ? shape[2] : 1;
  const int64_t npts = nx * ny * nz;
  const double inv_dx = 1.0 / dx;
#pragma omp parallel for schedule(static)
  for (int64_t p = 0; p < npts; ++p) {
    const int64_t k = p % nz, j = (p / nz) % ny, i = p / (nz * ny);
    int64_t np_[3], nm_[3];
    np_[0] = (wrap_p(i, nx) * ny + j) * nz + k;
    nm_[0] = (wrap_m(i, nx) * ny + j) * nz + k;
    np_[1] = (i * ny + wrap_p(j, ny)) * nz + k;
    nm_[1] = (i * ny + wrap_m(j, ny)) * nz + k;
    np_[2] = (i * ny + j) * nz + wrap_p(k, nz);
    nm_[2] = (i * ny + j) * nz + wrap_m(k, nz);
    for (int d = 0; d < dim; ++d)
      for (int s = 0; s < S; ++s) {
        const double center = c[p * c_stride + s];
        gp[(d * npts + p) * S + s] = (c[np_[d] * c_stride + s] - center) * inv_dx;
        gm[(d * npts + p) * S + s] = (center - c[nm_[d] * c_stride + s]) * inv_dx;
      }
  }
}

/* Face fluxes from stored gradients, (dim, *sp, S) outputs
 * (phasefield5d/solver/fluxes.py:26-125). */
PF5D_ORACLE_API void orc_fluxes_pm(int dim, const int64_t *shape, int S, const double *X,
                                   const double *M, int64_t m_stride, const double *gp,
                                   const double *gm, double *fp, double *fm) {
  int64_t nx = shape[0], ny = dim > 1 ? shape[1] : 1, nz = dim > 2 ? shape[2] : 1;
  const int64_t npts = nx * ny * nz;
#pragma omp parallel for schedule(static)
  for (int64_t p = 0; p < npts; ++p) {
    const int64_t k = p % nz, j = (p / nz) % ny, i = p / (nz * ny);
    int64_t np_[3], nm_[3];
    np_[0] = (wrap_p(i, nx) * ny + j) * nz + k;
    nm_[0] = (wrap_m(i, nx) * ny + j) * nz + k;
    np_[1] = (i * ny + wrap_p(j, ny)) * nz + k;
    nm_[1] = (i * ny + wrap_m(j, ny)) * nz + k;
    np_[2] = (i * ny + j) * nz + wrap_p(k, nz);
    nm_[2] = (i * ny + j) * nz + wrap_m(k, nz);
    for (int d = 0; d < dim; ++d) {
      const int64_t o = (d * npts + p) * S;
      face_flux(S, X + p * S, M + p * m_stride, X + np_[d] * S, M + np_[d] * m_stride, gp + o,
                fp + o);
      face_flux(S, X + p * S, M + p * m_stride, X + nm_[d] * S, M + nm_[d] * m_stride, gm + o,
                fm + o);
    }
  }
}

/* --------------------------------------------------------------------------
 * Reductions and update (operators.py:161-175, 262-317; simulate.py:315-317)
 * ------------------------------------------------------------------------ */

/* max |a[i]| starting from 0.0; NaN never wins (v > m is false). */
PF5D_ORACLE_API double orc_abs_max(const double *a, int64_t n) {
  double m = 0.0;
  for (int64_t i = 0; i < n; ++i) {
    const double v = fabs(a[i]);
    if (v > m) m = v;
  }
  return m;
}

/* Renormalise points with sum_s X[p,s] > 1 by multiplying with 1/total. */
PF5D_ORACLE_API void orc_clamp_simplex(double *X, int64_t npts, int S) {
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < npts; ++i) {
    double total = 0.0;
    for (int s = 0; s < S; ++s) total += X[i * S + s];
    if (total > 1.0) {
      const double inv = 1.0 / total;
      for (int s = 0; s < S; ++s) X[i * S + s] *= inv;
    }
  }
}

/* dXdt *= dt; X += dXdt (two roundings, simulate.py:316-317). */
PF5D_ORACLE_API void orc_update(double *X, double *dXdt, int64_t n, double dt) {
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) {
    dXdt[i] = dXdt[i] * dt;
    X[i] = X[i] + dXdt[i];
  }
}

PF5D_ORACLE_API int orc_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}
