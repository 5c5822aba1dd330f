"""Host-side logic of the serving loop with a fake device backend (no GPU):
admission by free HBM, step blocks that never pass a request's step count,
retirement of finished and halted requests, cancellation, statistics."""
import numpy as np
import pytest

from phasefield5d_b200.serving import Request, Scheduler, poisson_arrivals


class FakeProblem:
    def __init__(self, shape):
        self.shape = shape

    @property
    def dim(self):
        return len(self.shape)

    @property
    def n_points(self):
        return int(np.prod(self.shape))


class FakeBackend:
    def __init__(self, free):
        self.free = free
        self.active = []
        self.steps = {}
        self.halt_at = {}
        self.syncs = 0
        self.blocks = []

    def free_bytes(self):
        used = sum(r.device_bytes() for r in self.active)
        return self.free - used

    def sync(self, active):
        self.active = list(active)
        self.syncs += 1
        for r in active:
            self.steps.setdefault(r.rid, 0)

    def advance(self, blocks):
        self.blocks.append(dict(blocks))
        for rid, n in blocks.items():
            self.steps[rid] += n

    def states(self):
        out = {}
        for r in self.active:
            halted = r.rid in self.halt_at and self.steps[r.rid] >= self.halt_at[r.rid]
            out[r.rid] = {"step": self.steps[r.rid], "halted": halted, "dt": 1.0, "time": 0.0}
        return out

    def collect(self, req):
        return np.zeros(1)


class FakeClock:
    def __init__(self):
        self.t = 0.0

    def __call__(self):
        self.t += 0.001
        return self.t


def make(rid, shape, steps, arrival=0.0):
    return Request(rid=rid, problem=FakeProblem(shape), n_steps=steps, arrival=arrival)


def test_admission_limited_by_free_hbm():
    r0, r1, r2 = make(0, (4096,), 100), make(1, (4096,), 100), make(2, (4096,), 100)
    per = r0.device_bytes()
    be = FakeBackend(free=(1 << 20) + per * 2)
    sch = Scheduler(be, reserve_bytes=1 << 20, clock=FakeClock())
    for r in (r0, r1, r2):
        sch.submit(r)
    sch.tick()
    assert [r.rid for r in sch.active] == [0, 1]          # third does not fit
    assert [r.rid for r in sch.queue] == [2]
    sch.run()
    assert all(r.status == "done" for r in sch.finished) and len(sch.finished) == 3


def test_slot_limit_and_arrival_order():
    be = FakeBackend(free=1 << 40)
    sch = Scheduler(be, max_slots=2, reserve_bytes=0, clock=FakeClock())
    for i in range(5):
        sch.submit(make(i, (64, 64), 60, arrival=0.0))
    sch.tick()
    assert len(sch.active) == 2
    st = sch.run()
    assert st["requests_done"] == 5


def test_blocks_never_pass_step_counts():
    be = FakeBackend(free=1 << 40)
    sch = Scheduler(be, step_block=50, reserve_bytes=0, clock=FakeClock())
    reqs = [make(0, (4096,), 120), make(1, (64, 64), 75), make(2, (16, 16, 16), 130)]
    for r in reqs:
        sch.submit(r)
    sch.run()
    for r in reqs:
        assert be.steps[r.rid] == r.n_steps
    for b in be.blocks:                                    # shared group moves in lockstep
        shared = {b[k] for k in (0, 1) if k in b}
        assert len(shared) <= 1


def test_halted_request_retires_others_continue():
    be = FakeBackend(free=1 << 40)
    be.halt_at[1] = 10
    sch = Scheduler(be, step_block=10, reserve_bytes=0, clock=FakeClock())
    for r in (make(0, (256,), 40), make(1, (256,), 40)):
        sch.submit(r)
    st = sch.run()
    status = {r.rid: r.status for r in sch.finished}
    assert status == {0: "done", 1: "halted"}
    assert st["requests_halted"] == 1 and st["requests_done"] == 1


def test_cancel_queued_and_active():
    be = FakeBackend(free=1 << 40)
    sch = Scheduler(be, max_slots=1, step_block=5, reserve_bytes=0, clock=FakeClock())
    for r in (make(0, (256,), 100), make(1, (256,), 100)):
        sch.submit(r)
    sch.tick()
    assert sch.cancel(1)                                   # queued
    assert sch.cancel(0)                                   # active
    assert not sch.active and not sch.queue
    assert {r.status for r in sch.finished} == {"cancelled"}


def test_poisson_arrivals_rate():
    t = poisson_arrivals(20.0, 4000, seed=1)
    assert np.all(np.diff(t) > 0)
    assert t[-1] / 4000 == pytest.approx(1 / 20.0, rel=0.1)


class AsyncFakeBackend(FakeBackend):
    """Asynchronous protocol: the shared batch (dim < 3) and each 3D request
    are units; a unit's block takes `cost` polls per grid point-step."""

    def __init__(self, free, cost=1e-4):
        super().__init__(free)
        self.cost = cost
        self.inflight = {}      # unit -> [polls left, {rid: steps}]

    def shares_batch(self, r):
        return r.dim < 3

    def _unit(self, rid):
        r = next(r for r in self.active if r.rid == rid)
        return "batch" if r.dim < 3 else rid

    def busy(self):
        out = set()
        for unit in self.inflight:
            out.update(r.rid for r in self.active if self._unit(r.rid) == unit)
        return out

    def launch(self, blocks):
        self.blocks.append(dict(blocks))
        for rid, n in blocks.items():
            unit = self._unit(rid)
            work = self.inflight.setdefault(unit, [0, {}])
            r = next(r for r in self.active if r.rid == rid)
            work[0] += max(1, int(self.cost * n * r.n_points))
            work[1][rid] = n

    def poll(self, timeout):
        out = {}
        for unit in list(self.inflight):
            work = self.inflight[unit]
            work[0] -= 1
            if work[0] <= 0:
                del self.inflight[unit]
                for rid, n in work[1].items():
                    self.steps[rid] += n
                states = self.states()
                out.update({rid: states[rid] for rid in work[1] if rid in states})
        return out


def test_async_units_progress_independently():
    """A small request admitted after a large 3D one finishes first: units
    take their next block as soon as their own last block is done."""
    be = AsyncFakeBackend(free=1 << 40)
    sch = Scheduler(be, step_block=50, reserve_bytes=0, clock=FakeClock())
    big = make(0, (64, 64, 64), 400)
    small = make(1, (1024,), 400, arrival=0.0)
    mid = make(2, (64, 64), 300, arrival=0.0)
    for r in (big, small, mid):
        sch.submit(r)
    st = sch.run()
    assert st["requests_done"] == 3
    for r in (big, small, mid):
        assert be.steps[r.rid] == r.n_steps
    order = [r.rid for r in sorted(sch.finished, key=lambda r: r.done)]
    assert order.index(0) == 2                      # the 3D request finishes last
    for b in be.blocks:                             # batch members move in lockstep
        shared = {b[k] for k in (1, 2) if k in b}
        assert len(shared) <= 1
