"""Serving form: a continuous-batching solve server on one GPU.

Requests (a ``workload.Problem`` plus a step count) arrive over time.  The
server admits them while batch slots and free HBM allow, keeps their fields
and the temperature tables resident on the device, and advances them in
step blocks on device units that run independently -- each unit takes its
next block as soon as its own last one is done, so a small request is never
held by a large one's block:

* 1D and 2D solves share one batched stepper (``batch.BatchStepper``), one
  unit.  When a request joins, the batch is rebuilt and every continuing
  solve resumes its exact FP32 state (hi/lo pair, dt, time, step), so a
  request's trajectory does not depend on when others come and go.  When
  requests only leave (finished, halted, cancelled), the batch keeps
  running with the departed solves advancing unobserved, until the next
  join or until they are half the batch -- a rebuild per departure would
  stall the device units;
* 3D solves each get their own FP32-compensated ``Stepper`` on their own
  stream (one unit each), so their work overlaps the batch on the device;
* the device tables of each temperature are built once and shared by the
  batch and the 3D steppers.

``GpuBackend(precision="fp64")`` is the plain-FP64 comparison: every request
gets its own bit-faithful FP64 ``Stepper`` on its own stream (the FP64 form
has no batched kernel), with the same admission and step blocks.

A step block never takes a solve past its requested step count.  Each
finished request records its time to solution (arrival to result on the
host); ``stats()`` gives p50/p99 and the aggregate grid-point steps/s.

Scheduling (``Scheduler``) is separate from the device work (``GpuBackend``)
so the admission and block logic can be exercised with a fake backend.
"""
from __future__ import annotations

import time
from dataclasses import dataclass, field

import numpy as np

# Device bytes per grid point of an admitted FP32-compensated solve: hi, lo
# and dX/dt (3 x 16), the mu/M buffer of the split rate kernels (36), the
# misfit scalar and its half spectrum (~4 + 8), and working room for cuFFT
# (16).
BYTES_PER_POINT = 132
# The plain FP64 form: X and dX/dt (2 x 32), the mu/M buffer (72), the FP64
# misfit scalar and its half spectrum (8 + 16), cuFFT working room (32).
BYTES_PER_POINT_FP64 = 192
FIXED_BYTES_PER_SOLVE = 4 << 20


@dataclass
class Request:
    rid: int
    problem: object
    n_steps: int
    arrival: float = 0.0
    status: str = "queued"          # queued, active, done, halted, cancelled
    admitted: float | None = None
    done: float | None = None
    steps_done: int = 0
    result: np.ndarray | None = None
    final_state: dict | None = None

    @property
    def dim(self):
        return self.problem.dim

    @property
    def n_points(self):
        return int(self.problem.n_points)

    @property
    def remaining(self):
        return self.n_steps - self.steps_done

    def device_bytes(self, bytes_per_point=BYTES_PER_POINT):
        return bytes_per_point * self.n_points + FIXED_BYTES_PER_SOLVE


class Scheduler:
    """Admission, step blocks and retirement, independent of the device.

    ``backend`` provides: ``sync(active)`` (make the device set match the
    active requests), ``collect(req)`` (host field), ``free_bytes()``, and
    either the asynchronous pair ``launch(blocks)`` / ``poll(timeout)`` with
    ``busy()`` -- each device unit (the shared batch, each own stepper)
    takes its next block as soon as its last one is done, and ``poll``
    returns the states of the units that finished -- or the synchronous pair
    ``advance(blocks)`` / ``states()``, where every block waits for all.
    """

    def __init__(self, backend, max_slots=64, step_block=50, reserve_bytes=1 << 30,
                 clock=time.perf_counter):
        self.backend = backend
        self.max_slots = int(max_slots)
        self.step_block = int(step_block)
        self.reserve = int(reserve_bytes)
        self.clock = clock
        self.t0 = None
        self.queue: list[Request] = []
        self.active: list[Request] = []
        self.finished: list[Request] = []
        self.points_steps = 0

    def now(self):
        if self.t0 is None:
            self.t0 = self.clock()
        return self.clock() - self.t0

    def submit(self, req: Request):
        self.queue.append(req)
        self.queue.sort(key=lambda r: r.arrival)

    def cancel(self, rid):
        for r in list(self.queue):
            if r.rid == rid:
                self.queue.remove(r)
                r.status = "cancelled"
                self.finished.append(r)
                return True
        for r in list(self.active):
            if r.rid == rid:
                self.active.remove(r)
                r.status = "cancelled"
                r.done = self.now()
                self.finished.append(r)
                self.backend.sync(self.active)
                return True
        return False

    def admit(self):
        """Admit arrived requests in arrival order while slots and HBM allow."""
        now = self.now()
        admitted = []
        free = self.backend.free_bytes()
        for r in list(self.queue):
            if r.arrival > now or len(self.active) >= self.max_slots:
                break
            need = r.device_bytes(getattr(self.backend, "bytes_per_point", BYTES_PER_POINT))
            if free - need < self.reserve:
                break                       # head-of-line: keep arrival order
            self.queue.remove(r)
            r.status, r.admitted = "active", now
            self.active.append(r)
            admitted.append(r)
            free -= need
        return admitted

    def block_sizes(self):
        """Steps each active request advances this block: the step block, cut
        so no request of the shared batch (they move in lockstep) passes its
        count."""
        in_batch = getattr(self.backend, "shares_batch", lambda r: r.dim < 3)
        shared = [r for r in self.active if in_batch(r)]
        n_shared = min([self.step_block] + [r.remaining for r in shared]) if shared else 0
        return {r.rid: (n_shared if in_batch(r) else min(self.step_block, r.remaining))
                for r in self.active}

    def tick(self):
        """One scheduling iteration; returns False when nothing is left."""
        changed = bool(self.admit())
        if changed:
            self.backend.sync(self.active)
        if not self.active:
            if not self.queue:
                return False
            wait = self.queue[0].arrival - self.now()
            if wait > 0:
                time.sleep(min(wait, 0.01))
            return True
        if hasattr(self.backend, "launch"):
            busy = self.backend.busy()
            blocks = {rid: n for rid, n in self.block_sizes().items()
                      if n > 0 and rid not in busy}
            self.backend.launch(blocks)
            wait = 0.005
            if self.queue:
                wait = min(wait, max(self.queue[0].arrival - self.now(), 0.0))
            states = self.backend.poll(wait)
        else:
            self.backend.advance(self.block_sizes())
            states = self.backend.states()
        retired = False
        for r in list(self.active):
            if r.rid not in states:
                continue
            st = states[r.rid]
            self.points_steps += r.n_points * (st["step"] - r.steps_done)
            r.steps_done = st["step"]
            if st["halted"] or r.steps_done >= r.n_steps:
                r.status = "halted" if st["halted"] else "done"
                r.final_state = st
                r.result = self.backend.collect(r)
                r.done = self.now()
                self.active.remove(r)
                self.finished.append(r)
                retired = True
        if retired:
            self.backend.sync(self.active)
        return True

    def run(self, timeout=None):
        start = self.now()
        while self.tick():
            if timeout is not None and self.now() - start > timeout:
                break
        return self.stats()

    def stats(self):
        done = [r for r in self.finished if r.status == "done"]
        tts = np.array([r.done - r.arrival for r in done]) if done else np.array([np.nan])
        span = (max(r.done for r in done) - min(r.arrival for r in done)) if done else np.nan
        return {
            "requests_done": len(done),
            "requests_halted": sum(r.status == "halted" for r in self.finished),
            "requests_cancelled": sum(r.status == "cancelled" for r in self.finished),
            "p50_time_to_solution_s": float(np.percentile(tts, 50)),
            "p99_time_to_solution_s": float(np.percentile(tts, 99)),
            "grid_point_steps_per_s": float(self.points_steps / span) if done else float("nan"),
            "wall_s": float(span),
        }


class GpuBackend:
    """Device side of the server.  ``precision="fp32c"``: one batch for the
    1D/2D requests, one FP32-compensated stepper per 3D request.
    ``precision="fp64"``: one plain FP64 stepper per request."""

    def __init__(self, device=0, precision="fp32c"):
        import torch
        if precision not in ("fp32c", "fp64"):
            raise ValueError(f"unknown precision {precision!r}")
        self.precision = precision
        self.bytes_per_point = BYTES_PER_POINT if precision == "fp32c" else BYTES_PER_POINT_FP64
        from .batch import BatchStepper
        from .stepper import Stepper
        self.torch = torch
        self.BatchStepper = BatchStepper
        self.Stepper = Stepper
        torch.cuda.set_device(device)
        self.batch = None
        self.batch_ids: list[int] = []
        self.steppers: dict[int, object] = {}
        self.streams: dict[int, object] = {}
        self.reqs: dict[int, Request] = {}
        self.batch_stream = torch.cuda.Stream()
        self.variants: dict[tuple, int] = {}      # shape -> autotuned kernel variant
        self.tables: dict[tuple, object] = {}     # resident device tables, per temperature
        self.table_mu: dict[tuple, object] = {}   # mu reference each FP32 table subtracts
        self.pending: dict[object, object] = {}   # unit ("batch" or rid) -> event of its block
        self.fresh = False                        # batch rebuilt: report its states
        self.live: set[int] = set()               # batch solves still active

    def _table(self, prob):
        """Resident device table of the request's temperature (built once):
        FP32 mu - mu(equiatomic) for the compensated form -- the same table
        the batch uses -- or the padded FP64 table."""
        import numpy as np
        from .batch import TABLE_REFERENCE_X, _table32
        from .solver.table import host_table_eval
        from .stepper import device_table
        key = (prob.cfg.temperature, prob.table.seed, prob.cfg.resolution)
        if self.precision == "fp64":
            key = ("fp64",) + key
            if key not in self.tables:
                self.tables[key] = device_table(prob.grid, self.torch)
            return self.tables[key], None
        if key not in self.table_mu:
            self.table_mu[key] = host_table_eval(np.asarray(TABLE_REFERENCE_X)[None, :], prob.grid,
                                                 prob.cfg.resolution)[0, :4]
        if key not in self.tables:
            self.tables[key] = _table32(prob.grid, self.table_mu[key], self.torch)
        return self.tables[key], self.table_mu[key]

    def shares_batch(self, req):
        """True when the request advances in the shared 1D/2D batch."""
        return self.precision == "fp32c" and req.dim < 3

    def free_bytes(self):
        free, _total = self.torch.cuda.mem_get_info()
        return int(free)

    def sync(self, active):
        torch = self.torch
        ids = [r.rid for r in active]
        self.reqs = {r.rid: r for r in active}
        for rid in list(self.steppers):
            if rid not in ids:
                self.streams[rid].synchronize()
                self.steppers.pop(rid).close()
                self.streams.pop(rid)
                self.pending.pop(rid, None)
        for r in active:
            if not self.shares_batch(r) and r.rid not in self.steppers:
                s = torch.cuda.Stream()
                key = tuple(r.problem.shape)
                tab, mu0 = self._table(r.problem)
                with torch.cuda.stream(s):
                    st = self.Stepper.from_problem(r.problem, precision=self.precision, stream=s,
                                                   autotune=key not in self.variants, table=tab,
                                                   table_mu0=mu0)
                    if key in self.variants:
                        st.set_variant(self.variants[key])
                    else:
                        self.variants[key] = st.variant
                self.steppers[r.rid] = st
                self.streams[r.rid] = s
        want = [r.rid for r in active if self.shares_batch(r)]
        if want == self.batch_ids:
            return
        if (self.batch is not None and all(rid in self.batch_ids for rid in want)
                and 2 * len(want) >= len(self.batch_ids)):
            # Only retirements: the batch keeps running.  A retired solve (its
            # result already collected) advances unobserved until the next
            # rebuild, which saves a rebuild per retirement; the live solves'
            # trajectories do not depend on it.
            self.live = set(want)
            return
        resume = {}
        if self.batch is not None:
            with torch.cuda.stream(self.batch_stream):
                for k, rid in enumerate(self.batch_ids):
                    if rid in want:
                        resume[rid] = self.batch.export(k)
            self.batch_stream.synchronize()
            self.batch.close()
            self.batch = None
            self.pending.pop("batch", None)
        self.batch_ids = want
        self.live = set(want)
        if want:
            with torch.cuda.stream(self.batch_stream):
                self.batch = self.BatchStepper([self.reqs[i].problem for i in want],
                                               stream=self.batch_stream, autotune=False,
                                               resume=[resume.get(i) for i in want],
                                               table_cache=self.tables)
            self.fresh = True

    # -- asynchronous protocol: every unit runs its own blocks -------------
    def busy(self):
        """Request ids whose unit has a block not yet reported by poll."""
        out = set()
        for unit in self.pending:
            if unit == "batch":
                out.update(self.batch_ids)
            else:
                out.add(unit)
        return out

    def _batch_block(self, blocks):
        """Steps of the next batch block: the live solves move in lockstep."""
        return max([blocks.get(rid, 0) for rid in self.batch_ids if rid in self.live] + [0])

    def launch(self, blocks):
        torch = self.torch
        if self.batch is not None and self.batch_ids and "batch" not in self.pending:
            n = self._batch_block(blocks)
            if n > 0:
                self.batch.advance(n)
                ev = torch.cuda.Event()
                ev.record(self.batch_stream)
                self.pending["batch"] = ev
        for rid, st in self.steppers.items():
            n = blocks.get(rid, 0)
            if n > 0 and rid not in self.pending:
                st.advance(n)
                ev = torch.cuda.Event()
                ev.record(self.streams[rid])
                self.pending[rid] = ev

    def poll(self, timeout):
        """States of the units whose block finished (waits up to `timeout`
        seconds for the first one)."""
        deadline = time.perf_counter() + timeout
        while True:
            out = {}
            if self.fresh and self.batch is not None and "batch" not in self.pending:
                out.update(zip(self.batch_ids, self.batch.states()))
            self.fresh = False
            for unit, ev in list(self.pending.items()):
                if not ev.query():
                    continue
                del self.pending[unit]
                if unit == "batch":
                    out.update(zip(self.batch_ids, self.batch.states()))
                else:
                    out[unit] = self.steppers[unit].state()
            if out or time.perf_counter() >= deadline:
                return out
            time.sleep(0.0002)

    # -- synchronous protocol (every block waits for all units) -------------
    def advance(self, blocks):
        if self.batch is not None and self.batch_ids:
            n = self._batch_block(blocks)
            if n > 0:
                self.batch.advance(n)
        for rid, st in self.steppers.items():
            if blocks.get(rid, 0) > 0:
                st.advance(blocks[rid])
        self.torch.cuda.synchronize()

    def states(self):
        out = {}
        if self.batch is not None:
            for rid, st in zip(self.batch_ids, self.batch.states()):
                out[rid] = st
        for rid, st in self.steppers.items():
            out[rid] = st.state()
        return out

    def collect(self, req):
        if req.rid in self.steppers:
            return self.steppers[req.rid].field().cpu().numpy()
        k = self.batch_ids.index(req.rid)
        return self.batch.field(k).cpu().numpy()


class Server(Scheduler):
    """Scheduler + GPU backend."""

    def __init__(self, device=0, precision="fp32c", **kw):
        super().__init__(GpuBackend(device, precision), **kw)


# ---------------------------------------------------------------------------
# Request streams
# ---------------------------------------------------------------------------

def poisson_arrivals(rate, n, seed=0):
    """Arrival times (s) of n requests of a Poisson process of `rate` req/s."""
    rng = np.random.default_rng(seed)
    return np.cumsum(rng.exponential(1.0 / rate, size=n))


def serving_configs(n, seed=0, steps=2000, sizes_3d=(64, 96, 128, 160, 192)):
    """The serving mix: 1D 4096, 2D 256^2 and 3D 64^3-192^3 requests (equal
    shares), random compositions, kappa log-uniform in [1e-16, 1e-14], one
    of the four temperature tables, `steps` adaptive steps each."""
    from .workload import BATCH_TEMPERATURES, SolveConfig, random_composition
    rng = np.random.default_rng(seed)
    cfgs = []
    for i in range(n):
        kind = i % 3
        shape = [(4096,), (256, 256), None][kind]
        if shape is None:
            m = int(rng.choice(sizes_3d))
            shape = (m, m, m)
        cfgs.append(SolveConfig(
            system_dim=len(shape), initial_composition=random_composition(rng),
            kappa_value=float(10 ** rng.uniform(-16, -14)), resolution=0.025,
            temperature=BATCH_TEMPERATURES[int(rng.integers(0, 4))], shape=shape, adaptive=True,
            total_timesteps=steps, ic_seed=1000 + i, n_k=2000))
    return cfgs
