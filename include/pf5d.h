/*
 * pf5d.h -- C ABI of the B200 (sm_100a) Cahn-Hilliard step library.
 *
 * One shared library, libpf5d.so, built from phasefield5d_b200/csrc.  All
 * entry points take plain pointers and sizes; device pointers are CUDA
 * global-memory addresses on the current device, and `stream` is a
 * cudaStream_t passed as void* (NULL = legacy default stream).  Arrays use
 * the reference layout: C-contiguous (*spatial, S) float64 with S = 4
 * independent components; "views" (mu = interp[..., :4], M = interp[..., 4:])
 * are a pointer plus a point stride in elements.
 *
 * Every function returns a pf5d_status (0 = success).  Launch-only entry
 * points do not synchronise; errors found on the device are reported through
 * the device status word documented at PF5D_FLAG_*.  pf5d_last_error() gives
 * a text for the last non-zero return on the calling thread.
 *
 * Reference interfaces are cited as path:line within phasefield5d.
 */
#ifndef PF5D_H
#define PF5D_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Every declaration below is an exported symbol of libpf5d.so (the library
 * is built with hidden visibility by default). */
#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

/* ---------------------------------------------------------------- status */
typedef enum {
  PF5D_OK = 0,
  PF5D_ERR_ARG = 1,          /* bad pointer/size/stride (reference: ValueError)        */
  PF5D_ERR_DIM = 2,          /* unsupported spatial dimension (ValueError /
                                NotImplementedError in the reference)                   */
  PF5D_ERR_CUDA = 3,         /* a CUDA runtime call failed                             */
  PF5D_ERR_CUFFT = 4,        /* a cuFFT call failed                                    */
  PF5D_ERR_NN_DISTANCE = 5,  /* nearest table row farther than max_nn_dist
                                (reference: RuntimeError, interpolation.py:207-208)   */
  PF5D_ERR_OOB = 6,          /* hard out-of-bounds composition (system.py:12-53)       */
  PF5D_ERR_CAPACITY = 7      /* request exceeds a fixed capacity of the library        */
} pf5d_status;

/* Device status word bits (OR-ed by kernels). */
#define PF5D_FLAG_NONFINITE    0x01u  /* NaN/inf in the composition field           */
#define PF5D_FLAG_OOB_HARD     0x02u  /* |violation| > tol_hard (1e-3)              */
#define PF5D_FLAG_OOB_SOFT     0x04u  /* |violation| > tol_soft (1e-5)              */
#define PF5D_FLAG_NN_FAR       0x08u  /* nearest-row distance > max_nn_dist         */
#define PF5D_FLAG_NN_TRUNCATED 0x10u  /* nearest-row search found no present node   */
#define PF5D_FLAG_NN_USED      0x20u  /* some point took the nearest-row fallback   */
#define PF5D_FLAG_HALTED       0x40u  /* step loop stopped (OOB check or an NN error) */
#define PF5D_FLAG_NN_NONFINITE 0x80u  /* a fallback point had a NaN/inf component   */
/* The nearest-row search is exact for every finite point (it widens its
 * window until the nearest present node is proven).  NN_FAR, NN_TRUNCATED and
 * NN_NONFINITE are errors where the reference raises (RuntimeError for the
 * distance, ValueError from cKDTree.query for a non-finite point): the step
 * loop halts before that step's update, and the Python mirror raises. */

const char *pf5d_last_error(void);
int32_t pf5d_version(void);

/* ------------------------------------------------------- interpolation ----
 * interpolator_nb (phasefield5d/solver/interpolation.py:154-211):
 * quadrilinear interpolation of a dense (n,n,n,n,node_stride) table with the
 * nearest-table-row fallback for points with sum(x) > 1 - 4*res - 1e-9.
 * comp: device (npts,4); grid: device dense table, props at [0, nprops) of
 * each node's node_stride values, NaN at nodes absent from the table;
 * node_coord: device (n,) stored coordinate of node k on every axis;
 * out: device, row r at out + r*out_stride; mask: device (npts,) bytes or
 * NULL; flags: device uint32 OR-ed with PF5D_FLAG_NN_* or NULL.
 * max_nn_dist <= 0 disables the distance check. */
pf5d_status pf5d_interp4d(const double *comp, int64_t npts, const double *grid, int32_t n,
                          int32_t nprops, int32_t node_stride, double resolution,
                          const double *node_coord, double max_nn_dist, double *out,
                          int64_t out_stride, uint8_t *mask, uint32_t *flags, void *stream);

/* ----------------------------------------------------------- stencils -----
 * calculate_laplacian (phasefield5d/solver/operators.py:10-76): periodic
 * second-order Laplacian of a contiguous (*shape, ncomp) field. */
pf5d_status pf5d_laplacian(int32_t dim, const int64_t *shape, int32_t ncomp, const double *c,
                           double dx, double *out, void *stream);

/* lap *= kappa; mu -= lap  (examples/simulate.py:254-255).  kappa: host (ncomp,). */
pf5d_status pf5d_kappa_subtract(double *mu, int64_t mu_stride, double *lap, const double *kappa,
                                int64_t npts, int32_t ncomp, void *stream);

/* get_divergence_from_mu_function(dim)(X, M, mu, inv_dx, out)
 * (phasefield5d/solver/fluxes.py:296-416, face flux 128-160). */
pf5d_status pf5d_divergence_from_mu(int32_t dim, const int64_t *shape, int32_t ncomp,
                                    const double *X, const double *M, int64_t m_stride,
                                    const double *mu, int64_t mu_stride, double inv_dx,
                                    double *out, void *stream);

/* calculate_gradients_pm (phasefield5d/solver/operators.py:79-123, 126-158,
 * 289-317): gp, gm device (dim, *shape, ncomp). */
pf5d_status pf5d_gradients_pm(int32_t dim, const int64_t *shape, int32_t ncomp, const double *c,
                              int64_t c_stride, double dx, double *gp, double *gm, void *stream);

/* get_flux_function(dim)(X, M, gp, gm, fp, fm)
 * (phasefield5d/solver/fluxes.py:6-125). */
pf5d_status pf5d_fluxes_pm(int32_t dim, const int64_t *shape, int32_t ncomp, const double *X,
                           const double *M, int64_t m_stride, const double *gp, const double *gm,
                           double *fp, double *fm, void *stream);

/* ------------------------------------------------------------ elastic -----
 * make_elastic_updater (phasefield5d/solver/elastic.py:147-286), rank-1 path:
 * s = (X - X0).l ; S = rfftn(s) * B(k) ; s' = irfftn(S) ; mu += s' l.
 * bk: host real B(k) on the rfft half-grid (copied at create).  One cuFFT
 * D2Z/Z2D plan pair per handle. */
typedef struct pf5d_elastic pf5d_elastic;
pf5d_status pf5d_elastic_create(int32_t dim, const int64_t *shape, const double *x0,
                                const double *lvec, const double *bk, pf5d_elastic **out);
pf5d_status pf5d_elastic_apply(pf5d_elastic *h, double *mu, int64_t mu_stride, const double *X,
                               void *stream);
pf5d_status pf5d_elastic_destroy(pf5d_elastic *h);

/* --------------------------------------------------------- reductions -----
 * abs_max (phasefield5d/solver/operators.py:161-175): max |a[i]| starting
 * from 0.0, NaN ignored.  result: device double.  Uses a per-device block
 * partials workspace allocated on first use. */
pf5d_status pf5d_abs_max(const double *a, int64_t n, double *result, void *stream);

/* No counterpart in the reference.  The same reduction as pf5d_abs_max for
 * callers that cannot allow a library to allocate device memory (a host
 * whose own pool owns the GPU's memory, or a loop that must not risk the
 * synchronisation cudaMalloc/cudaFree can cause).  Its scratch is a fixed
 * 256 KiB __device__ array held by every GPU that loads the library, so the
 * call allocates nothing; n is limited to 67,108,864 elements (larger n is
 * rejected with PF5D_ERR_CAPACITY).  The first call on a device looks up
 * that array's device address (cudaGetSymbolAddress); make that first call
 * before any stream capture.  Calls share the array: calls whose kernels
 * overlap on the GPU race. */
pf5d_status pf5d_abs_max_noalloc(const double *a, int64_t n, double *result, void *stream);

/* clamp_simplex (phasefield5d/solver/operators.py:262-317), in place. */
pf5d_status pf5d_clamp_simplex(double *X, int64_t npts, int32_t ncomp, void *stream);

/* dXdt *= dt; X += dXdt  (examples/simulate.py:316-317). */
pf5d_status pf5d_update(double *X, double *dXdt, int64_t n, double dt, void *stream);

/* out_of_bounds statistics (phasefield5d/solver/system.py:12-53).  Fills
 * host stats[5] = {n_nonfinite, max row sum, min row sum, max comp, min comp}
 * (synchronises `stream`). */
pf5d_status pf5d_oob_stats(const double *X, int64_t npts, int32_t ncomp, double *stats,
                           void *stream);

/* apply_adaptive_time (phasefield5d/solver/system.py:90-112) on the host;
 * the step loop evaluates the same rule on the device. */
double pf5d_adaptive_dt(double dt_current, double xdotmax, double ctld, double t_cfl,
                        double lower_limit, double upper_limit, double max_change_factor);

/* ---------------------------------------------------------- step loop -----
 * The main loop body of examples/simulate.py:230-320 (saves off) as a
 * device-resident stepper: interpolation, Laplacian, elastic term, fused
 * flux divergence, max|dX/dt|, adaptive dt, update and clamp, with dt and
 * time kept on the device and steps replayed from CUDA graphs.  The
 * out_of_bounds check runs every oob_interval steps before the step, as in
 * simulate.py:231; a hard violation halts the stepper (PF5D_FLAG_HALTED). */
typedef struct {
  int32_t dim;                 /* 1, 2 or 3                                   */
  int64_t shape[3];            /* cells per axis (unused trailing = 1)        */
  double dx;                   /* cell size [m]                               */
  double kappa[4];             /* kappa_i * kappa_value per component         */
  double x0[4];                /* reference composition                        */
  int32_t elastic;             /* 1: rank-1 Khachaturyan term on             */
  double lvec[4];              /* rank-1 factor l (Lambda = l l^T)            */
  const double *bk;            /* host B(k) on the rfft half-grid, or NULL    */
  const double *grid;          /* device dense table (caller owns)            */
  int32_t table_n;             /* nodes per axis                              */
  int32_t nprops;              /* 9                                           */
  int32_t node_stride;         /* doubles per node (>= nprops)               */
  double resolution;           /* table spacing                               */
  const double *node_coord;    /* device (table_n,)                           */
  double max_nn_dist;          /* <= 0: unchecked                             */
  double ctld, t_cfl;          /* CTLD [s] and CFL bound [s]                  */
  double lower_limit, upper_limit, max_change_factor;
  int32_t adaptive;            /* 0: fixed dt = dt0                           */
  double dt0;                  /* initial dt                                  */
  int32_t oob_interval;        /* 100 in the reference                        */
  int32_t precision;           /* PF5D_PRECISION_FP64 or _FP32C                */
  const float *grid32;         /* FP32C: device table, node_stride32 floats per
                                  node: mu - mu0 (4), M (5), pad               */
  int32_t node_stride32;       /* 12                                          */
  double mu0[4];               /* FP32C: mu at X0 subtracted from the table   */
} pf5d_stepper_desc;

/* Precision forms of the stepper.  FP64: bit-faithful to the reference
 * (apart from FFT rounding); X is advanced in place.  FP32C: D = X - X0 as
 * an FP32 hi/lo pair with a compensated update, FP32 stencils, table and
 * FFT, FP64 closure / sums / dt / mass; X only seeds the state (read it back
 * with pf5d_stepper_field). */
#define PF5D_PRECISION_FP64 0
#define PF5D_PRECISION_FP32C 1

typedef struct {
  double dt, time, xdotmax;
  int64_t step;
  uint32_t flags;
  uint32_t halted;
} pf5d_step_state;

typedef struct pf5d_stepper pf5d_stepper;

/* X: device (*shape, 4) float64, caller-owned, advanced in place. */
pf5d_status pf5d_stepper_create(const pf5d_stepper_desc *desc, double *X, void *stream,
                                pf5d_stepper **out);
/* Enqueue n steps on `stream` (no host synchronisation). */
pf5d_status pf5d_stepper_advance(pf5d_stepper *h, int64_t nsteps, void *stream);
/* Synchronise `stream` and copy the device step state to *out. */
pf5d_status pf5d_stepper_state(pf5d_stepper *h, pf5d_step_state *out, void *stream);
/* Device pointer to the last dX/dt buffer ((*shape, 4); float64 for FP64,
 * float32 for FP32C). */
double *pf5d_stepper_rate(pf5d_stepper *h);
/* Write the current field X ((*shape, 4) float64, device) to X_out. */
pf5d_status pf5d_stepper_field(pf5d_stepper *h, double *X_out, void *stream);
/* FP64 mean composition per component (host mean_out[4]); synchronises.
 * The mass-drift report is its change over a run. */
pf5d_status pf5d_stepper_mass(pf5d_stepper *h, double *mean_out, void *stream);
/* Diagnostics: launch one stage of a step by itself on `stream`
 * (PF5D_STAGE_*), so each kernel can be timed with events.  It changes the
 * stepper's state exactly as that stage does inside a step. */
#define PF5D_STAGE_RATE 0        /* rate kernel(s) (mu/M + flux divergence) and the dt controller */
#define PF5D_STAGE_UPDATE 1      /* update, clamp, next misfit, OOB test       */
#define PF5D_STAGE_FFT_FWD 2     /* cuFFT D2Z of the misfit (2D with a power-of-two
                                    axis 0 up to 1024: the row D2Z); 1D solves up to
                                    16384 points: the whole elastic term in closed form */
#define PF5D_STAGE_BMUL 3        /* B(k) multiply (2D column pass: axis-0 transform,
                                    multiply, inverse; nothing in the 1D closed form) */
#define PF5D_STAGE_FFT_INV 4     /* cuFFT Z2D (2D column pass: the row Z2D; nothing in
                                    the 1D closed form)                          */
pf5d_status pf5d_stepper_launch_stage(pf5d_stepper *h, int32_t stage, void *stream);
/* Autotuner: time every rate-kernel variant (plane tile shape x resident
 * blocks per SM, ...) on this solve; the plain FP64 form then times the
 * fastest few as captured graphs of whole steps and keeps the fastest.  The
 * field and step state are preserved.  *variant / *best_ms (either may be
 * NULL) report the choice and its time: ms per step (plain FP64 2D/3D) or
 * ms per rate stage (other forms). */
pf5d_status pf5d_stepper_autotune(pf5d_stepper *h, int32_t *variant, float *best_ms,
                                  void *stream);
/* Select a rate-kernel variant explicitly (index from a previous autotune). */
pf5d_status pf5d_stepper_set_variant(pf5d_stepper *h, int32_t variant);
/* Save-step diagnostics of one step (examples/simulate.py:299-354): the
 * values the reference records in its traces at a save step.  "Before" values
 * use the step's dX/dt before it is scaled by dt; "after" values use the
 * field after the update and clamp. */
typedef struct {
  double net[4];            /* before: sum over space of dX/dt */
  double max_change[4];     /* before: max over space of |dX/dt| per component */
  double total_flux[4];     /* before: sum over space and axes of flux_p - flux_m */
  double mass[4];           /* after: sum over space of X */
  double comp_min[4];       /* after: min over space of X */
  double comp_max[4];       /* after: max over space of X */
  double comp_fe_min;       /* after: 1 - max over space of sum_s X_s */
  double comp_var[4];       /* after: variance over space of X (population) */
  double f_grad;            /* after: -(dx^dim / 2) sum X . kappa lap X */
  double xdotmax;           /* the step's max |dX/dt| (abs_max) */
  double dt;                /* the step's time increment */
  double time;              /* time after the step */
  int64_t step;             /* index of this step (count before it) */
  int32_t halted;           /* 1: the stepper was halted before; nothing ran */
  int32_t pad;
} pf5d_save_diag;

/* One step, exactly as pf5d_stepper_advance(h, 1), plus the save-step
 * diagnostics of that step; synchronises the stream.  Replaces the save
 * branch of examples/simulate.py:299-354 (calculate_gradients_pm,
 * compute_fluxes and the numpy reductions).  Either form; the FP32C form
 * reduces FP64 copies of its field X0 + hi + lo, dX/dt and mu/M. */
pf5d_status pf5d_stepper_step_save(pf5d_stepper *h, pf5d_save_diag *out, void *stream);
/* Number of rate-kernel variants of this stepper's form (valid indices for
 * pf5d_stepper_set_variant are 0 .. count-1); 0 for a null stepper. */
int32_t pf5d_stepper_variant_count(const pf5d_stepper *h);
/* Kernels of this library that one step launches with the current variant
 * (rate kernel(s), dt controller, update, and when elasticity is on the B(k)
 * multiply -- the column kernel in 2D with a power-of-two axis 0, the
 * closed-form kernel in 1D; cuFFT's own kernels not counted); 0 for a null
 * stepper. */
int32_t pf5d_stepper_launches_per_step(const pf5d_stepper *h);
/* The kernel instances one rate stage of the current variant launches, as
 * profilers name them ("k_rate_tile2d<32, 8, 2, 1, 1, 0, 352, 1, 0> +
 * k_dt_finish"); the text is owned by the stepper and valid until the next
 * call on it.  No counterpart in the reference (a diagnostic). */
const char *pf5d_stepper_rate_kernels(pf5d_stepper *h);
/* Re-derive internal state after the caller modified X (e.g. a restart). */
pf5d_status pf5d_stepper_reset(pf5d_stepper *h, double dt, double time, void *stream);
pf5d_status pf5d_stepper_destroy(pf5d_stepper *h);

/* ------------------------------------------------------- batched form -----
 * Many independent FP32-compensated 1D/2D solves advanced together: one
 * persistent rate launch over the tiles of all solves, one compensated-update
 * launch, cuFFT plans batched per 2D shape; each solve keeps its own
 * adaptive dt.  This replaces the reference's one-process-per-solve sweeps
 * (run/launch.py:119-150) with one device-resident batch. */
typedef struct {
  int32_t dim;                 /* 1 or 2                                      */
  int64_t shape[2];
  double dx;
  double kappa[4];
  double x0[4];
  int32_t elastic;
  double lvec[4];
  const double *bk;            /* host B(k) on the rfft half-grid            */
  int32_t table;               /* index into the batch's FP32 tables         */
  double max_nn_dist;
  double ctld, t_cfl, lower_limit, upper_limit, max_change_factor;
  int32_t adaptive;
  double dt0;
  int32_t oob_interval;
  const double *X;             /* device (*shape, 4) float64 initial field   */
  /* Optional exact resume (continuous batching): when hi / lo are not NULL
   * they seed X - X0 as the FP32 pair (device, 4 floats per point each)
   * instead of X, and time0 / step0 seed the step state (dt from dt0). */
  const float *hi, *lo;
  double time0;
  int64_t step0;
} pf5d_batch_solve;

typedef struct pf5d_batch pf5d_batch;

/* tables32: device FP32 tables (12 floats per node: mu - mu_ref (4), M (5),
 * pad), all with table_n nodes per axis and the given resolution. */
pf5d_status pf5d_batch_create(const pf5d_batch_solve *solves, int32_t nsolves,
                              const float *const *tables32, int32_t ntables, int32_t table_n,
                              double resolution, const double *node_coord, void *stream,
                              pf5d_batch **out);
pf5d_status pf5d_batch_advance(pf5d_batch *h, int64_t nsteps, void *stream);
/* out: nsolves entries; synchronises `stream`. */
pf5d_status pf5d_batch_states(pf5d_batch *h, pf5d_step_state *out, void *stream);
pf5d_status pf5d_batch_field(pf5d_batch *h, int32_t i, double *X_out, void *stream);
/* Copy solve i's FP32 pair (X - X0 = hi + lo; device, 4 floats per point
 * each) for an exact resume in another batch. */
pf5d_status pf5d_batch_export(pf5d_batch *h, int32_t i, float *hi_out, float *lo_out, void *stream);
pf5d_status pf5d_batch_autotune(pf5d_batch *h, int32_t *variant, float *best_ms, void *stream);
pf5d_status pf5d_batch_set_variant(pf5d_batch *h, int32_t variant);
/* Number of batched rate-kernel variants (valid indices 0 .. count-1). */
int32_t pf5d_batch_variant_count(void);
pf5d_status pf5d_batch_destroy(pf5d_batch *h);

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif

#ifdef __cplusplus
}
#endif
#endif /* PF5D_H */
