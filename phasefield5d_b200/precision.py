"""Accuracy report of the FP32-compensated form against the plain FP64 form.

Both forms run on the GPU from the same initial field for the same number
of steps; the report gives the max and RMS error of X (relative to max|X|)
and of X - X0 (relative to max|X64 - X0|, the stricter measure), plus each
form's mass drift (change of the FP64 mean composition per component).
"""
from __future__ import annotations

import numpy as np

from .stepper import Stepper


def compare_forms(prob, n_steps, chunk=500, **kw):
    """Run ``n_steps`` in both forms; return the report dict."""
    a = Stepper.from_problem(prob, precision="fp64", **kw)
    b = Stepper.from_problem(prob, precision="fp32c", **kw)
    m64_0, m32_0 = a.mass(), b.mass()
    done = 0
    while done < n_steps:
        n = min(chunk, n_steps - done)
        a.advance(n)
        b.advance(n)
        done += n
    sa, sb = a.state(), b.state()
    x64 = a.field().cpu().numpy()
    x32 = b.field().cpu().numpy()
    m64_1, m32_1 = a.mass(), b.mass()
    a.close()
    b.close()
    return report(x64, x32, prob.X0, sa, sb, m64_1 - m64_0, m32_1 - m32_0, n_steps)


def report(x64, x32, X0, s64, s32, drift64, drift32, n_steps):
    err = np.abs(x32 - x64)
    dev = np.abs(x64 - np.asarray(X0))
    scale_x = float(np.max(np.abs(x64)))
    scale_dev = max(float(np.max(dev)), 1e-300)
    return {
        "steps": int(n_steps),
        "max_rel_err_X": float(np.max(err)) / scale_x,
        "rms_rel_err_X": float(np.sqrt(np.mean(err ** 2))) / scale_x,
        "max_rel_err_X_minus_X0": float(np.max(err)) / scale_dev,
        "rms_rel_err_X_minus_X0": float(np.sqrt(np.mean(err ** 2))) / scale_dev,
        "mass_drift_fp32c": [float(v) for v in drift32],
        "mass_drift_fp64": [float(v) for v in drift64],
        "time_fp64": s64["time"], "time_fp32c": s32["time"],
        "dt_fp64": s64["dt"], "dt_fp32c": s32["dt"],
        "halted": bool(s64["halted"] or s32["halted"]),
    }
