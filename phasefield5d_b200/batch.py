"""Batched form: many independent FP32-compensated 1D/2D solves advanced
together by the batched CUDA stepper (``pf5d_batch_*``).

This is the in-process replacement for the reference's one-process-per-solve
parameter sweeps (run/launch.py:119-150): every solve of the batch shares
each launch of a step, keeps its own adaptive dt, and reads one of a few
temperature tables resident in HBM.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from .solver.table import host_table_eval
from .stepper import NODE_STRIDE32


def _table32(grid, mu_ref, torch):
    g = np.asarray(grid)[..., :9].astype(np.float64)
    out = np.zeros((*g.shape[:-1], NODE_STRIDE32), dtype=np.float32)
    out[..., :4] = (g[..., :4] - np.asarray(mu_ref)).astype(np.float32)
    out[..., 4:9] = g[..., 4:9].astype(np.float32)
    return torch.from_numpy(out).cuda()


# Reference composition whose mu each FP32 table subtracts: the equiatomic
# point of the five species.  It is fixed per table, so a solve's table (and
# its trajectory) does not depend on which other solves share the batch.
TABLE_REFERENCE_X = (0.2, 0.2, 0.2, 0.2)


class BatchStepper:
    """Advance a list of ``workload.Problem`` (1D/2D, same table resolution)
    together.  Problems with the same temperature share one device table,
    which stores mu - mu(TABLE_REFERENCE_X) and M in FP32."""

    def __init__(self, problems, stream=None, autotune=True, oob_interval=100, resume=None,
                 table_cache=None):
        """``resume[i]`` (optional): ``(hi, lo, dt, time, step)`` from
        ``export(j)`` of another batch -- solve i then continues that state
        exactly instead of starting from ``problems[i].X_init``.
        ``table_cache`` (optional dict): device tables kept across batches,
        keyed by (temperature, table seed, resolution); a batch rebuilt for
        new membership then reuses the resident tables."""
        import torch
        self._torch = torch
        self.L = _lib.load()
        self.stream = stream
        self.problems = list(problems)
        res = {p.cfg.resolution for p in self.problems}
        if len(res) != 1:
            raise ValueError("all solves of a batch must use one table resolution")
        self.resolution = res.pop()
        keys = []
        for p in self.problems:
            k = (p.cfg.temperature, p.table.seed)
            if k not in keys:
                keys.append(k)
        self.table_keys = keys
        self.tables = []
        cache = table_cache if table_cache is not None else {}
        for k in keys:
            ck = (*k, self.resolution)
            if ck not in cache:
                grid = next(p for p in self.problems
                            if (p.cfg.temperature, p.table.seed) == k).grid
                mu_ref = host_table_eval(np.asarray(TABLE_REFERENCE_X)[None, :], grid,
                                         self.resolution)[0, :4]
                cache[ck] = _table32(grid, mu_ref, torch)
            self.tables.append(cache[ck])
        self.node_coord = torch.from_numpy(np.ascontiguousarray(self.problems[0].node_coord)).cuda()
        resume = list(resume) if resume is not None else [None] * len(self.problems)
        self._resume = resume
        self.X_init = [None if r is not None else
                       torch.from_numpy(np.ascontiguousarray(p.X_init)).cuda()
                       for p, r in zip(self.problems, resume)]
        self._bk = []
        arr = (_lib.BatchSolve * len(self.problems))()
        for i, p in enumerate(self.problems):
            q = arr[i]
            q.dim = p.dim
            for d in range(2):
                q.shape[d] = p.shape[d] if d < p.dim else 1
            q.dx = p.dx
            kap = np.asarray(p.kappa, dtype=np.float64).reshape(-1)
            elastic = p.lvec is not None and p.bk is not None
            for c in range(4):
                q.kappa[c] = float(kap[c])
                q.x0[c] = float(p.X0[c])
                q.lvec[c] = float(p.lvec[c]) if elastic else 0.0
            q.elastic = 1 if elastic else 0
            if elastic:
                bk = np.ascontiguousarray(p.bk, dtype=np.float64)
                self._bk.append(bk)
                q.bk = bk.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
            q.table = keys.index((p.cfg.temperature, p.table.seed))
            q.max_nn_dist = -1.0
            q.ctld, q.t_cfl = p.ctld, p.t_cfl
            q.lower_limit, q.upper_limit = p.cfg.lower_limit, p.cfg.upper_limit
            q.max_change_factor = 2.0
            q.adaptive = 1 if p.cfg.adaptive else 0
            q.dt0 = p.dt0
            q.oob_interval = int(oob_interval)
            r = resume[i]
            if r is None:
                q.X = self.X_init[i].data_ptr()
            else:
                hi, lo, dt, time, step = r
                q.hi, q.lo = hi.data_ptr(), lo.data_ptr()
                q.dt0, q.time0, q.step0 = float(dt), float(time), int(step)
        tabs = (ctypes.c_void_p * len(self.tables))(*[t.data_ptr() for t in self.tables])
        h = ctypes.c_void_p()
        _lib.check(self.L.pf5d_batch_create(arr, len(self.problems), tabs, len(self.tables),
                                            int(self.problems[0].grid.shape[0]), self.resolution,
                                            _lib.ptr(self.node_coord), self._s(), ctypes.byref(h)),
                   "BatchStepper")
        self.h = h
        self._arr = arr
        self.variant, self.tuned_ms = (self.autotune() if autotune else (0, None))

    def _s(self):
        return _lib.stream_handle(self.stream)

    @property
    def n_points(self):
        return int(sum(p.n_points for p in self.problems))

    def advance(self, n_steps):
        _lib.check(self.L.pf5d_batch_advance(self.h, int(n_steps), self._s()), "advance")

    def states(self):
        """Per-solve step state, with the nearest-row fallback bits decoded
        as in ``Stepper.state`` (a solve whose fallback failed is halted)."""
        out = (_lib.StepState * len(self.problems))()
        _lib.check(self.L.pf5d_batch_states(self.h, out, self._s()), "states")
        return [dict(dt=s.dt, time=s.time, xdotmax=s.xdotmax, step=int(s.step),
                     flags=int(s.flags), halted=bool(s.halted), **_lib.nn_flags(int(s.flags)))
                for s in out]

    def field(self, i):
        p = self.problems[i]
        out = self._torch.empty((*p.shape, 4), dtype=self._torch.float64, device="cuda")
        _lib.check(self.L.pf5d_batch_field(self.h, int(i), _lib.ptr(out), self._s()), "field")
        return out

    def export(self, i):
        """(hi, lo, dt, time, step) of solve i for an exact resume elsewhere."""
        p = self.problems[i]
        hi = self._torch.empty((p.n_points, 4), dtype=self._torch.float32, device="cuda")
        lo = self._torch.empty_like(hi)
        _lib.check(self.L.pf5d_batch_export(self.h, int(i), _lib.ptr(hi), _lib.ptr(lo), self._s()),
                   "export")
        st = self.states()[i]
        return hi, lo, st["dt"], st["time"], st["step"]

    def autotune(self):
        v = ctypes.c_int32()
        ms = ctypes.c_float()
        _lib.check(self.L.pf5d_batch_autotune(self.h, ctypes.byref(v), ctypes.byref(ms), self._s()),
                   "autotune")
        return int(v.value), float(ms.value)

    @property
    def n_variants(self):
        """Number of batched rate-kernel variants the autotuner chooses from."""
        return int(self.L.pf5d_batch_variant_count())

    def set_variant(self, v):
        _lib.check(self.L.pf5d_batch_set_variant(self.h, int(v)), "set_variant")

    def close(self):
        if getattr(self, "h", None):
            self.L.pf5d_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
