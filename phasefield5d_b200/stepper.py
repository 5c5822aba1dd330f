"""Device-resident step loop (examples/simulate.py:230-320 with saves off).

``Stepper`` owns the composition field on the GPU and advances it with the
fused CUDA step of ``libpf5d.so``: dt, time and the step counter stay on the
device, steps are replayed from CUDA graphs, and the host only reads the
state when asked.  The out-of-bounds test runs every ``oob_interval`` steps
before the step, exactly where the reference driver runs it, and a hard
violation halts the stepper with the field left as the reference leaves it.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib


class Stepper:
    """Stepper for one solve, in the plain FP64 form (bit-faithful to the
    reference up to FFT rounding; advances ``X`` in place) or the
    FP32-compensated form (``precision="fp32c"``: X - X0 as an FP32 hi/lo
    pair, FP32 stencils/table/FFT, FP64 closure/sums/dt; read the field with
    ``field()``).

    Parameters mirror the reference driver's state: dense table ``grid``
    (n,n,n,n,9) with its ``resolution`` and per-axis ``node_coord``; initial
    field ``X`` (*shape, 4); ``X0``; per-component ``kappa``; cell size
    ``dx``; rank-1 elastic factor ``lvec`` and ``bk`` = B(k) on the rfft
    half-grid (both None: elasticity off); ``ctld``, ``t_cfl``, initial
    ``dt``; ``adaptive`` (False: dt fixed); change limits.

    ``table`` (optional): the device table already in the layout of this
    form -- (n,n,n,n,10) float64 for "fp64", (n,n,n,n,12) float32 holding
    mu - ``table_mu0`` for "fp32c" -- so solves at the same temperature can
    share one resident copy.
    """

    def __init__(self, *, grid, resolution, node_coord, X, X0, kappa, dx, lvec, bk, ctld, t_cfl,
                 dt, adaptive=True, lower_limit=1e-5, upper_limit=1e-3, max_change_factor=2.0,
                 oob_interval=100, max_nn_dist=None, stream=None, autotune=True,
                 precision="fp64", table=None, table_mu0=None):
        import torch
        self._torch = torch
        self.L = _lib.load()
        self.stream = stream
        X = np.asarray(X, dtype=np.float64) if not isinstance(X, torch.Tensor) else X
        self.shape = tuple(int(s) for s in X.shape[:-1])
        self.dim = len(self.shape)
        if self.dim not in (1, 2, 3):
            raise ValueError(f"Unsupported system_dim={self.dim}. Choose 1, 2, or 3.")
        if precision not in ("fp64", "fp32c"):
            raise ValueError(f"precision must be 'fp64' or 'fp32c' (got {precision!r})")
        self.precision = precision
        if table is not None and precision == "fp32c" and table_mu0 is None:
            raise ValueError("a shared FP32 table needs the mu reference it subtracts (table_mu0)")
        if precision == "fp64":
            self.grid = table if table is not None else device_table(grid, torch)
            table_n = int(self.grid.shape[0])
        else:
            self.grid = None
            table_n = int(table.shape[0]) if table is not None else int(np.shape(grid)[0])
        self.node_coord = torch.from_numpy(np.ascontiguousarray(node_coord,
                                                                dtype=np.float64)).cuda()
        if isinstance(X, torch.Tensor):
            self.X = X.to(device="cuda", dtype=torch.float64).contiguous().clone()
        else:
            self.X = torch.from_numpy(np.ascontiguousarray(X)).cuda()
        elastic = lvec is not None and bk is not None
        d = _lib.StepperDesc()
        d.dim = self.dim
        for i, s in enumerate(self.shape):
            d.shape[i] = s
        for i in range(self.dim, 3):
            d.shape[i] = 1
        d.dx = float(dx)
        kap = np.asarray(kappa, dtype=np.float64).reshape(-1)
        for i in range(4):
            d.kappa[i] = float(kap[i])
            d.x0[i] = float(X0[i])
            d.lvec[i] = float(lvec[i]) if elastic else 0.0
        d.elastic = 1 if elastic else 0
        self._bk = np.ascontiguousarray(bk, dtype=np.float64) if elastic else None
        d.bk = (self._bk.ctypes.data_as(ctypes.POINTER(ctypes.c_double)) if elastic
                else ctypes.POINTER(ctypes.c_double)())
        d.grid = self.grid.data_ptr() if self.grid is not None else None
        d.table_n = table_n
        d.nprops = 9
        d.node_stride = int(self.grid.shape[-1]) if self.grid is not None else NODE_STRIDE
        d.resolution = float(resolution)
        d.node_coord = self.node_coord.data_ptr()
        d.max_nn_dist = float(max_nn_dist) if max_nn_dist is not None else -1.0
        d.ctld = float(ctld)
        d.t_cfl = float(t_cfl)
        d.lower_limit = float(lower_limit)
        d.upper_limit = float(upper_limit)
        d.max_change_factor = float(max_change_factor)
        d.adaptive = 1 if adaptive else 0
        d.dt0 = float(dt)
        d.oob_interval = int(oob_interval)
        d.precision = _lib.PRECISION_FP64 if precision == "fp64" else _lib.PRECISION_FP32C
        if precision == "fp32c":
            if table is not None:
                mu0, self.grid32 = np.asarray(table_mu0, dtype=np.float64), table
            else:
                mu0 = reference_mu(grid, resolution, X0)
                self.grid32 = device_table32(grid, mu0, torch)
            d.grid32 = self.grid32.data_ptr()
            d.node_stride32 = NODE_STRIDE32
            for i in range(4):
                d.mu0[i] = float(mu0[i])
        self.desc = d
        h = ctypes.c_void_p()
        _lib.check(self.L.pf5d_stepper_create(ctypes.byref(d), _lib.ptr(self.X), self._s(),
                                              ctypes.byref(h)), "Stepper")
        self.h = h
        self.steps_enqueued = 0
        self.variant, self.tuned_ms = (self.autotune() if autotune else (0, None))

    @classmethod
    def from_problem(cls, prob, **kw):
        """Stepper for a ``phasefield5d_b200.workload.Problem``."""
        return cls(grid=prob.grid, resolution=prob.cfg.resolution, node_coord=prob.node_coord,
                   X=prob.X_init, X0=prob.X0, kappa=prob.kappa, dx=prob.dx, lvec=prob.lvec,
                   bk=prob.bk, ctld=prob.ctld, t_cfl=prob.t_cfl, dt=prob.dt0,
                   adaptive=prob.cfg.adaptive, lower_limit=prob.cfg.lower_limit,
                   upper_limit=prob.cfg.upper_limit, **kw)

    def _s(self):
        return _lib.stream_handle(self.stream)

    @property
    def n_points(self):
        return int(np.prod(self.shape))

    def advance(self, n_steps):
        """Enqueue ``n_steps`` steps on the stream; returns without waiting."""
        _lib.check(self.L.pf5d_stepper_advance(self.h, int(n_steps), self._s()), "advance")
        self.steps_enqueued += int(n_steps)

    def state(self):
        """Synchronise and return {dt, time, xdotmax, step, flags, halted}
        plus the decoded nearest-row fallback bits: ``nn_used`` (some point
        took the fallback), ``nn_far`` (a row farther than max_nn_dist),
        ``nn_nonfinite`` (a non-finite composition reached the fallback) and
        ``nn_no_row``.  The last three halt the loop before that step's
        update, where the reference's loop raises."""
        st = _lib.StepState()
        _lib.check(self.L.pf5d_stepper_state(self.h, ctypes.byref(st), self._s()), "state")
        out = dict(dt=st.dt, time=st.time, xdotmax=st.xdotmax, step=int(st.step),
                   flags=int(st.flags), halted=bool(st.halted))
        out.update(_lib.nn_flags(int(st.flags)))
        return out

    def run(self, n_steps):
        """Advance ``n_steps`` and return the state; ``halted`` is True when an
        out-of-bounds check stopped the loop (simulate.py:231-239).  A
        nearest-row error raises as the reference's loop does: ValueError for
        a non-finite composition, RuntimeError for a row beyond max_nn_dist;
        the field is left as it was before the failing step."""
        self.advance(n_steps)
        st = self.state()
        if st["halted"]:
            _lib.raise_nn_errors(st["flags"])
        return st

    def rate(self):
        """dX/dt of the last step as a (*shape, 4) CUDA tensor (a view)."""
        ptr = self.L.pf5d_stepper_rate(self.h)
        return _tensor_from_ptr(ptr, self.n_points * 4, self._torch).view(*self.shape, 4)

    def autotune(self):
        """Pick the fastest rate-kernel variant for this solve (in-library
        autotuner); returns (variant index, ms per rate launch)."""
        v = ctypes.c_int32()
        ms = ctypes.c_float()
        _lib.check(self.L.pf5d_stepper_autotune(self.h, ctypes.byref(v), ctypes.byref(ms),
                                                self._s()), "autotune")
        return int(v.value), float(ms.value)

    def step_save(self):
        """One step plus its save-step diagnostics (examples/simulate.py:299-354),
        either form (the FP32-compensated one reduces its field X0 + hi + lo,
        dX/dt and mu/M in FP64): a dict with net, max_change, total_flux, mass,
        comp_min, comp_max, comp_var (arrays of 4), comp_fe_min, f_grad,
        xdotmax, dt, time (after the step), step (its index) and halted."""
        d = _lib.SaveDiag()
        _lib.check(self.L.pf5d_stepper_step_save(self.h, ctypes.byref(d), self._s()), "step_save")
        self.steps_enqueued += 0 if d.halted else 1
        out = {k: np.array(list(getattr(d, k))) for k in
               ("net", "max_change", "total_flux", "mass", "comp_min", "comp_max", "comp_var")}
        out.update(comp_fe_min=d.comp_fe_min, f_grad=d.f_grad, xdotmax=d.xdotmax, dt=d.dt,
                   time=d.time, step=int(d.step), halted=bool(d.halted))
        return out

    @property
    def launches_per_step(self):
        """Kernels of this library one step launches (cuFFT's not counted)."""
        return int(self.L.pf5d_stepper_launches_per_step(self.h))

    @property
    def rate_kernels(self):
        """The kernel instances one rate stage of the current variant launches
        (profiler names), e.g. for a roofline report."""
        return (self.L.pf5d_stepper_rate_kernels(self.h) or b"").decode()

    @property
    def n_variants(self):
        """Number of rate-kernel variants the autotuner chooses from."""
        return int(self.L.pf5d_stepper_variant_count(self.h))

    def set_variant(self, variant):
        _lib.check(self.L.pf5d_stepper_set_variant(self.h, int(variant)), "set_variant")

    def field(self):
        """Current field X as a (*shape, 4) float64 CUDA tensor (a copy)."""
        out = self._torch.empty((*self.shape, 4), dtype=self._torch.float64, device="cuda")
        _lib.check(self.L.pf5d_stepper_field(self.h, _lib.ptr(out), self._s()), "field")
        return out

    def mass(self):
        """FP64 mean composition per component (the quantity the flux form
        conserves; its change over a run is the mass drift)."""
        ptr, keep = _lib.f64_array([0.0] * 4)
        _lib.check(self.L.pf5d_stepper_mass(self.h, ptr, self._s()), "mass")
        return np.array(list(keep))

    def launch_stage(self, stage):
        """Diagnostics: enqueue one stage of a step (``_lib.STAGE_*``) alone."""
        _lib.check(self.L.pf5d_stepper_launch_stage(self.h, int(stage), self._s()), "stage")

    def reset(self, dt, time=0.0):
        """Re-read X (after the caller changed it) and restart dt/time/step."""
        _lib.check(self.L.pf5d_stepper_reset(self.h, float(dt), float(time), self._s()), "reset")

    def close(self):
        if getattr(self, "h", None):
            self.L.pf5d_stepper_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


NODE_STRIDE = 10
NODE_STRIDE32 = 12


def reference_mu(grid, resolution, X0):
    """mu(X0) from the FP64 table (quadrilinear, host): the shift the FP32
    table subtracts so it stores small deviations."""
    from .solver.table import host_table_eval
    g = grid.cpu().numpy() if hasattr(grid, "cpu") else np.asarray(grid)
    return host_table_eval(np.asarray(X0, dtype=np.float64)[None, :], g[..., :9], resolution)[0, :4]


def device_table32(grid, mu0, torch):
    """FP32 table, 12 floats per node (48-byte nodes, three float4 loads):
    mu - mu0 (4), M (5), pad.  Absent nodes stay NaN."""
    g = grid.cpu().numpy() if hasattr(grid, "cpu") else np.asarray(grid)
    g = g[..., :9].astype(np.float64)
    out = np.zeros((*g.shape[:-1], NODE_STRIDE32), dtype=np.float32)
    out[..., :4] = (g[..., :4] - np.asarray(mu0, dtype=np.float64)).astype(np.float32)
    out[..., 4:9] = g[..., 4:9].astype(np.float32)
    return torch.from_numpy(out).cuda()


def device_table(grid, torch):
    """Dense (n,n,n,n,9) table as a device tensor padded to 10 doubles per node
    (80-byte nodes: every node starts on a 16-byte boundary, so the fused
    kernels read each node as five double2 loads)."""
    if isinstance(grid, torch.Tensor):
        g = grid.to(device="cuda", dtype=torch.float64)
    else:
        g = torch.from_numpy(np.ascontiguousarray(grid, dtype=np.float64)).cuda()
    if g.shape[-1] == NODE_STRIDE:
        return g.contiguous()
    if g.shape[-1] != 9:
        raise ValueError(f"table must have 9 props per node (got {g.shape[-1]})")
    out = torch.zeros((*g.shape[:-1], NODE_STRIDE), dtype=torch.float64, device="cuda")
    out[..., :9] = g
    return out


def _tensor_from_ptr(ptr, n, torch):
    """Non-owning float64 CUDA tensor over ``n`` doubles at device address ptr."""
    class _Holder:
        pass
    h = _Holder()
    h.__cuda_array_interface__ = {"shape": (n,), "typestr": "<f8", "data": (int(ptr), False),
                                  "version": 3, "strides": None}
    return torch.as_tensor(h, device="cuda")
