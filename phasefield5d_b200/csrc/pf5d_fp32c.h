// pf5d_fp32c.h -- the FP32-compensated form of the step loop (internal).
//
// State: D = X - X0 kept as an unevaluated FP32 pair (hi, lo) per component
// and updated with a compensated (TwoSum) add, so the field carries ~48
// significant bits while every stencil, table lookup and FFT runs in FP32.
// FP64 is used only for the dependent-component closure X_Fe = 1 - sum X,
// the linear-region / simplex sums, the adaptive-dt controller, the k=0
// elastic mode (exactly zero: B(0) = 0) and the mean / mass reductions.
#pragma once

#include <cstdint>

#include "../../include/pf5d.h"

namespace pf5d {

struct Stepper32;

pf5d_status s32_create(const pf5d_stepper_desc *desc, const double *X_init, void *stream,
                       Stepper32 **out);
pf5d_status s32_advance(Stepper32 *h, int64_t nsteps, void *stream);
pf5d_status s32_state(Stepper32 *h, pf5d_step_state *out, void *stream);
pf5d_status s32_field(Stepper32 *h, double *X_out, void *stream);
pf5d_status s32_mass(Stepper32 *h, double *mean_out, void *stream);
pf5d_status s32_autotune(Stepper32 *h, int32_t *variant, float *best_ms, void *stream);
pf5d_status s32_set_variant(Stepper32 *h, int32_t variant);
int32_t s32_variant_count();
// Kernel instances of the current variant's rate stage (text owned by h).
const char *s32_rate_kernels(Stepper32 *h);
// Save steps: one step up to its rate evaluation plus FP64 copies of the
// field before the update (X), dX/dt and mu/M (SoA, 9 rows); then the update.
pf5d_status s32_step_save_inputs(Stepper32 *h, double *X_out, double *dX_out, double *mm_out,
                                 void *stream);
pf5d_status s32_step_update(Stepper32 *h, void *stream);
int32_t s32_launches_per_step(const Stepper32 *h);
pf5d_status s32_launch_stage(Stepper32 *h, int32_t stage, void *stream);
pf5d_status s32_reset(Stepper32 *h, const double *X, double dt, double time, void *stream);
float *s32_rate(Stepper32 *h);
void s32_destroy(Stepper32 *h);

}  // namespace pf5d
