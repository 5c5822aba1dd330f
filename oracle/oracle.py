"""CPU oracle for the phasefield5d step loop -- TEST INFRASTRUCTURE ONLY.

Imported only by ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline
leg of ``bench.py``, always as the checker.  The product (the CUDA library
and ``phasefield5d_b200``) never imports it.

The per-point kernels are the C restatement in ``pf5d_oracle.c`` (bit-faithful
to the reference's Numba kernels); the FFT pair is ``scipy.fft.rfftn/irfftn``
and the out-of-table fallback is ``scipy.spatial.cKDTree``, the same library
calls the reference makes.  ``OracleStepper.step`` runs one explicit step in
the order of examples/simulate.py:242-320 with saves off.

Parity status: pinned.  ``tests/golden/make_golden.py`` runs the reference
itself on seeded inputs and ``tests/test_oracle_golden.py`` requires this
oracle to reproduce those outputs bit for bit.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libpf5d_oracle.so")
_lib = None

_dp = ctypes.POINTER(ctypes.c_double)
_i64p = ctypes.POINTER(ctypes.c_int64)
_u8p = ctypes.POINTER(ctypes.c_uint8)


def build(force=False):
    """Compile pf5d_oracle.c with its Makefile (gcc, -ffp-contract=off)."""
    src = os.path.join(_HERE, "pf5d_oracle.c")
    if force or not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(src):
        subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(_LIB_PATH)
        L.orc_linear_mask.argtypes = [_dp, ctypes.c_int64, ctypes.c_int, ctypes.c_double, _u8p]
        L.orc_interp4d.argtypes = [_dp, ctypes.c_int64, _dp, ctypes.c_int, ctypes.c_int,
                                   ctypes.c_double, _dp, _u8p]
        L.orc_laplacian.argtypes = [ctypes.c_int, _i64p, ctypes.c_int, _dp, ctypes.c_double, _dp]
        L.orc_kappa_subtract.argtypes = [_dp, ctypes.c_int64, _dp, _dp, ctypes.c_int64, ctypes.c_int]
        L.orc_dot_misfit.argtypes = [_dp, ctypes.c_int64, ctypes.c_int, _dp, _dp, _dp]
        L.orc_expand_add.argtypes = [_dp, ctypes.c_int64, _dp, _dp, ctypes.c_int64, ctypes.c_int]
        L.orc_divergence_from_mu.argtypes = [ctypes.c_int, _i64p, ctypes.c_int, _dp, _dp,
                                             ctypes.c_int64, _dp, ctypes.c_int64,
                                             ctypes.c_double, _dp]
        L.orc_gradients_pm.argtypes = [ctypes.c_int, _i64p, ctypes.c_int, _dp, ctypes.c_int64,
                                       ctypes.c_double, _dp, _dp]
        L.orc_fluxes_pm.argtypes = [ctypes.c_int, _i64p, ctypes.c_int, _dp, _dp, ctypes.c_int64,
                                    _dp, _dp, _dp, _dp]
        L.orc_abs_max.argtypes = [_dp, ctypes.c_int64]
        L.orc_abs_max.restype = ctypes.c_double
        L.orc_clamp_simplex.argtypes = [_dp, ctypes.c_int64, ctypes.c_int]
        L.orc_update.argtypes = [_dp, _dp, ctypes.c_int64, ctypes.c_double]
        L.orc_num_threads.restype = ctypes.c_int
        _lib = L
    return _lib


def num_threads():
    return int(lib().orc_num_threads())


def _p(a, t=_dp):
    return a.ctypes.data_as(t)


def _shape(a):
    return np.asarray(a, dtype=np.int64)


def _view_stride(a):
    """Point stride (in elements) of a (*sp, S) view whose last axis is unit-stride."""
    assert a.strides[-1] == 8
    return a.strides[-2] // 8 if a.ndim >= 2 else a.shape[-1]


# ---------------------------------------------------------------------------
# Reference-named entry points (signatures of phasefield5d.solver.*)
# ---------------------------------------------------------------------------

def interpolator_nb(composition_array, data_grid, resolution, tree, calphad_values,
                    max_nn_dist=None, out=None, mask_buffer=None):
    """phasefield5d/solver/interpolation.py:154-211."""
    comp = np.ascontiguousarray(composition_array, dtype=np.float64)
    sp = comp.shape[:-1]
    n_props = data_grid.shape[4]
    if out is None:
        out = np.empty((*sp, n_props), dtype=np.float64)
    cf = comp.reshape(-1, 4)
    of = out.reshape(-1, n_props)
    mask = mask_buffer if mask_buffer is not None else np.empty(cf.shape[0], dtype=np.bool_)
    thr = 1.0 - 4.0 * resolution - 1e-9
    L = lib()
    grid = np.ascontiguousarray(data_grid, dtype=np.float64)
    L.orc_linear_mask(_p(cf), cf.shape[0], 4, thr, mask.ctypes.data_as(_u8p))
    L.orc_interp4d(_p(cf), cf.shape[0], _p(grid), grid.shape[0], n_props, float(resolution),
                   _p(of), mask.ctypes.data_as(_u8p))
    bad = ~mask
    if bad.any():
        dists, nn = tree.query(cf[bad])
        if max_nn_dist is not None and np.any(dists > max_nn_dist):
            raise RuntimeError("Some compositions are outside the CALPHAD domain (KD-tree).")
        of[bad] = calphad_values[nn]
    return out


def calculate_laplacian(array, cell_size, out=None):
    """phasefield5d/solver/operators.py:10-29."""
    a = np.ascontiguousarray(array, dtype=np.float64)
    if out is None:
        out = np.empty_like(a)
    dim = a.ndim - 1
    if dim not in (1, 2, 3):
        raise NotImplementedError(f"Laplacian not implemented for spatial_dims={dim}")
    lib().orc_laplacian(dim, _p(_shape(a.shape[:-1]), _i64p), a.shape[-1], _p(a),
                        float(cell_size), _p(out))
    return out


def get_divergence_from_mu_function(system_dim):
    """phasefield5d/solver/fluxes.py:398-416; returns f(X, M, mu, inv_dx, out)."""
    if system_dim not in (1, 2, 3):
        raise ValueError(f"Unsupported system_dim={system_dim}. Choose 1, 2, or 3.")

    def f(X, M, mu, inv_dx, out):
        assert X.flags.c_contiguous and out.flags.c_contiguous
        lib().orc_divergence_from_mu(system_dim, _p(_shape(X.shape[:-1]), _i64p), X.shape[-1],
                                     _p(X), M.ctypes.data_as(_dp), _view_stride(M),
                                     mu.ctypes.data_as(_dp), _view_stride(mu), float(inv_dx),
                                     _p(out))
    return f


def calculate_gradients_pm(array, cell_size, grad_p=None, grad_m=None):
    """phasefield5d/solver/operators.py:88-123 (save-step diagnostics)."""
    dim = array.ndim - 1
    sp = array.shape[:-1]
    S = array.shape[-1]
    if grad_p is None:
        grad_p = np.empty((dim, *sp, S))
    if grad_m is None:
        grad_m = np.empty_like(grad_p)
    lib().orc_gradients_pm(dim, _p(_shape(sp), _i64p), S, array.ctypes.data_as(_dp),
                           _view_stride(array), float(cell_size), _p(grad_p), _p(grad_m))
    return grad_p, grad_m


def compute_fluxes(X, M, gp, gm, fp, fm):
    """phasefield5d/solver/fluxes.py:26-125 (save-step diagnostics)."""
    dim = X.ndim - 1
    lib().orc_fluxes_pm(dim, _p(_shape(X.shape[:-1]), _i64p), X.shape[-1], _p(X),
                        M.ctypes.data_as(_dp), _view_stride(M), _p(gp), _p(gm), _p(fp), _p(fm))


def abs_max(arr):
    """phasefield5d/solver/operators.py:161-175."""
    a = np.ascontiguousarray(arr, dtype=np.float64).reshape(-1)
    return float(lib().orc_abs_max(_p(a), a.shape[0]))


def clamp_simplex(composition):
    """phasefield5d/solver/operators.py:304-317 (in place)."""
    assert composition.flags.c_contiguous
    lib().orc_clamp_simplex(_p(composition), composition.size // composition.shape[-1],
                            composition.shape[-1])


def apply_adaptive_time(dt_current, xdotmax, ctld, t_cfl, *, composition_change_lower_limit=1e-5,
                        composition_change_upper_limit=1e-3, max_change_factor=2.0):
    """phasefield5d/solver/system.py:90-112."""
    if xdotmax is None or xdotmax <= 0.0:
        dt_raw = dt_current
    else:
        lo = composition_change_lower_limit / xdotmax
        hi_b = composition_change_upper_limit / xdotmax
        if lo > hi_b:
            lo, hi_b = hi_b, lo
        dt_raw = float(np.clip(dt_current, lo, hi_b))
    hi = dt_current * max_change_factor
    dt_new = min(hi, dt_raw)
    return min(dt_new, 0.005 * ctld, t_cfl)


def out_of_bounds(composition, tol_soft=1e-5, tol_hard=1e-3):
    """phasefield5d/solver/system.py:12-53 (messages omitted)."""
    if not np.isfinite(composition).all():
        return True
    sums = composition.sum(axis=-1)
    return bool(sums.max() > 1.0 + tol_hard or sums.min() < 0.0 - tol_hard
                or composition.min() < 0.0 - tol_hard or composition.max() > 1.0 + tol_hard)


def make_elastic_updater(X0, lvec, elastic_kernel_r, field_shape, fft_workers=-1):
    """Rank-1 scipy path of phasefield5d/solver/elastic.py:242-263.

    Takes the rank-1 factor directly (the reference derives it from Λ with
    ``np.linalg.eigh``; the caller passes that same vector).
    """
    from scipy.fft import rfftn, irfftn
    sp = tuple(field_shape[:-1])
    S = field_shape[-1]
    axes = tuple(range(len(sp)))
    X0 = np.asarray(X0, dtype=np.float64)
    lvec = np.asarray(lvec, dtype=np.float64)
    work_r = np.empty(sp)
    work_k = np.empty(elastic_kernel_r.shape, dtype=np.complex128)
    L = lib()

    def elastic_update(mu, X):
        L.orc_dot_misfit(_p(X), work_r.size, S, _p(X0), _p(lvec), _p(work_r))
        work_k[...] = rfftn(work_r, axes=axes, workers=fft_workers)
        work_k[...] *= elastic_kernel_r
        sr = np.ascontiguousarray(irfftn(work_k, s=sp, axes=axes, workers=fft_workers).real)
        L.orc_expand_add(mu.ctypes.data_as(_dp), _view_stride(mu), _p(sr), _p(lvec), sr.size, S)
    return elastic_update


# ---------------------------------------------------------------------------
# Step loop (examples/simulate.py:230-320, saves off)
# ---------------------------------------------------------------------------

def run_simulation(ost, total_steps, path, *, ctld, t_cfl, early_stage_frames=100,
                   late_burst_duration_ctld=100, late_burst_frames=700, late_tail_frames=300,
                   oob_interval=100):
    """The main loop of examples/simulate.py:200-365 on an ``OracleStepper``:
    the out-of-bounds check every ``oob_interval`` steps, ``should_save``
    called every step with the time after it, state files and traces at
    data saves, the final state.  Returns (traces, files)."""
    from phasefield5d_b200.solver.io import (finalize_traces, init_traces,
                                             save_current_state, should_save, update_traces)
    kw = dict(early_frames=early_stage_frames, burst_duration_ctld=late_burst_duration_ctld,
              burst_frames=late_burst_frames, tail_dt_ctld=late_tail_frames, snapshot_factor=10)
    files = [save_current_state(path, 0, 0, 0.0, ost.X, postfix="_initial")]
    traces = init_traces(4)
    should_save._state = None
    timestep = 0
    for timestep in range(total_steps):
        if timestep % oob_interval == 0 and out_of_bounds(ost.X):
            files.append(save_current_state(path, timestep, ost.dt, ost.time, ost.X,
                                            postfix="_out_of_bound"))
            break
        d = ost.step_save()
        save_data, _ = should_save(timestep, ctld, d["time"], total_steps, **kw)
        if save_data:
            files.append(save_current_state(path, timestep, d["dt"], d["time"], ost.X))
            update_traces(traces, timestep, d["time"], d["dt"], t_cfl, d["net"], d["xdotmax"],
                          d["max_change"], d["mass"], d["total_flux"], d["comp_min"],
                          d["comp_max"], d["comp_fe_min"], d["comp_var"], d["f_grad"])
    files.append(save_current_state(path, timestep, ost.dt, ost.time, ost.X))
    finalize_traces(path, traces)
    return traces, files


class OracleStepper:
    """Explicit Euler loop of the reference driver on host arrays.

    Inputs are plain arrays/scalars: dense table ``grid`` (n,n,n,n,9),
    ``resolution``, KD-tree + row values for the fallback, ``X`` (*sp, 4),
    ``X0``, ``kappa`` (4,), ``dx``, ``lvec`` and ``bk`` (None = elasticity off),
    ``ctld``, ``t_cfl``, initial ``dt``, ``adaptive`` flag and the change limits.
    """

    def __init__(self, *, grid, resolution, tree, calphad_values, X, X0, kappa, dx, lvec, bk,
                 ctld, t_cfl, dt, adaptive=True, lower_limit=1e-5, upper_limit=1e-3,
                 fft_workers=-1):
        self.grid = np.ascontiguousarray(grid, dtype=np.float64)
        self.resolution = float(resolution)
        self.tree, self.values = tree, calphad_values
        self.X = np.array(X, dtype=np.float64, order="C", copy=True)
        self.sp = self.X.shape[:-1]
        self.dim = len(self.sp)
        self.kappa = np.asarray(kappa, dtype=np.float64).reshape(1, 4)
        self.dx = float(dx)
        self.inv_dx = 1.0 / self.dx
        self.ctld, self.t_cfl = float(ctld), float(t_cfl)
        self.dt = float(dt)
        self.adaptive = bool(adaptive)
        self.lower, self.upper = float(lower_limit), float(upper_limit)
        self.time = 0.0
        self.step_index = 0
        self.xdotmax = 0.0
        self.interp = np.empty((*self.sp, self.grid.shape[-1]))
        self.lap = np.empty_like(self.X)
        self.dXdt = np.empty_like(self.X)
        self.mask = np.empty(int(np.prod(self.sp)), dtype=np.bool_)
        self.div = get_divergence_from_mu_function(self.dim)
        self.elastic = None
        if lvec is not None and bk is not None:
            self.elastic = make_elastic_updater(X0, lvec, bk, self.X.shape, fft_workers)

    @classmethod
    def from_problem(cls, prob, fft_workers=-1):
        return cls(grid=prob.grid, resolution=prob.cfg.resolution, tree=prob.tree,
                   calphad_values=prob.calphad_values, X=prob.X_init, X0=prob.X0,
                   kappa=prob.kappa, dx=prob.dx, lvec=prob.lvec, bk=prob.bk, ctld=prob.ctld,
                   t_cfl=prob.t_cfl, dt=prob.dt0, adaptive=prob.cfg.adaptive,
                   lower_limit=prob.cfg.lower_limit, upper_limit=prob.cfg.upper_limit,
                   fft_workers=fft_workers)

    def compute_rate(self):
        """Steps 2-7 of the loop: returns dX/dt in self.dXdt and max|dX/dt|."""
        interpolator_nb(self.X, self.grid, self.resolution, self.tree, self.values,
                        out=self.interp, mask_buffer=self.mask)
        mu = self.interp[..., :4]
        M = self.interp[..., 4:]
        calculate_laplacian(self.X, self.dx, self.lap)
        lib().orc_kappa_subtract(mu.ctypes.data_as(_dp), _view_stride(mu), _p(self.lap),
                                 _p(np.ascontiguousarray(self.kappa.reshape(-1))),
                                 self.lap.size // 4, 4)
        if self.elastic is not None:
            self.elastic(mu, self.X)
        self.div(self.X, M, mu, self.inv_dx, self.dXdt)
        self.xdotmax = abs_max(self.dXdt)
        return self.xdotmax

    def step(self):
        self.compute_rate()
        if self.adaptive:
            self.dt = apply_adaptive_time(self.dt, self.xdotmax, self.ctld, self.t_cfl,
                                          composition_change_lower_limit=self.lower,
                                          composition_change_upper_limit=self.upper)
        self.time += self.dt
        lib().orc_update(_p(self.X), _p(self.dXdt), self.X.size, self.dt)
        clamp_simplex(self.X)
        self.step_index += 1

    def step_save(self):
        """One step with the save-step diagnostics of examples/simulate.py:299-354
        (numpy reductions in the reference's form).  ``flux_abs`` (the sum of
        |flux_p| + |flux_m|) is the scale of the total-flux rounding noise."""
        ax = tuple(range(self.dim))
        self.compute_rate()
        if self.adaptive:
            self.dt = apply_adaptive_time(self.dt, self.xdotmax, self.ctld, self.t_cfl,
                                          composition_change_lower_limit=self.lower,
                                          composition_change_upper_limit=self.upper)
        net = np.sum(self.dXdt, axis=ax)
        max_change = np.max(np.abs(self.dXdt), axis=ax)
        mu = np.ascontiguousarray(self.interp[..., :4])
        M = self.interp[..., 4:]
        gp, gm = calculate_gradients_pm(mu, self.dx)
        fp = np.empty_like(gp)
        fm = np.empty_like(gm)
        compute_fluxes(self.X, M, gp, gm, fp, fm)
        step = self.step_index
        self.time += self.dt
        lib().orc_update(_p(self.X), _p(self.dXdt), self.X.size, self.dt)
        clamp_simplex(self.X)
        self.step_index += 1
        lap = np.empty_like(self.X)
        calculate_laplacian(self.X, self.dx, lap)
        lap *= self.kappa
        return dict(
            net=net, max_change=max_change,
            total_flux=np.sum(fp - fm, axis=tuple(range(self.dim + 1))),
            flux_abs=float(np.sum(np.abs(fp)) + np.sum(np.abs(fm))),
            mass=np.sum(self.X, axis=ax), comp_min=np.min(self.X, axis=ax),
            comp_max=np.max(self.X, axis=ax),
            comp_fe_min=1.0 - float(np.max(self.X.sum(axis=-1))),
            comp_var=np.var(self.X, axis=ax),
            f_grad=-0.5 * (self.dx ** self.dim) * float(np.sum(self.X * lap)),
            xdotmax=self.xdotmax, dt=self.dt, time=self.time, step=step, halted=False)

    def run(self, n_steps, oob_interval=100):
        """Advance n_steps; stops early (returns False) on a hard OOB check,
        which runs every ``oob_interval`` steps before the step as in
        examples/simulate.py:231."""
        for _ in range(n_steps):
            if self.step_index % oob_interval == 0 and out_of_bounds(self.X):
                return False
            self.step()
        return True
