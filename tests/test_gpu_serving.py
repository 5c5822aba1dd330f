"""Serving loop on the GPU: continuous batching with requests arriving while
others run.  Each request's result is the same alone and in the mix: bit for
bit for 1D (shared batch, exact state transfer on every batch rebuild) and
3D (own stepper) requests, within the FP32c tolerance (1e-6 relative) for
2D requests (the cuFFT plan batch size changes with the mix)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FIELD_RTOL_FP32C = 1e-6


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _requests(steps=120):
    from phasefield5d_b200 import workload as W
    from phasefield5d_b200.serving import Request, serving_configs
    cfgs = serving_configs(6, seed=3, steps=steps, sizes_3d=(24, 32))
    shapes = [(1024,), (48, 48), (24, 24, 24), (2048,), (64, 64), (32, 32, 32)]
    probs = []
    for c, sh in zip(cfgs, shapes):
        c.shape, c.system_dim = sh, len(sh)
        probs.append(W.build_batched_problems([c])[0][0])
    return [Request(rid=i, problem=p, n_steps=steps + 10 * i) for i, p in enumerate(probs)]


def _serve(reqs, arrivals, **kw):
    from phasefield5d_b200.serving import Server
    srv = Server(step_block=kw.pop("step_block", 25), reserve_bytes=0, **kw)
    for r, a in zip(reqs, arrivals):
        r.arrival = a
        srv.submit(r)
    st = srv.run(timeout=300)
    return srv, st


def test_alone_equals_mix(torch_cuda):
    import copy
    reqs = _requests()
    _, st = _serve([copy.copy(r) for r in reqs], [0.0, 0.01, 0.02, 0.05, 0.08, 0.12])
    mixed = {r.rid: r for r in _.finished}
    assert st["requests_done"] == len(reqs)
    for r in reqs:
        srv, _st = _serve([copy.copy(r)], [0.0])
        alone = srv.finished[0]
        m = mixed[r.rid]
        assert alone.status == m.status == "done"
        assert alone.final_state["step"] == m.final_state["step"] == r.n_steps
        if r.dim in (1, 3):
            assert np.array_equal(alone.result, m.result), r.rid
            assert alone.final_state["time"] == m.final_state["time"]
        else:
            scale = np.max(np.abs(m.result))
            assert np.max(np.abs(alone.result - m.result)) <= FIELD_RTOL_FP32C * scale


def test_poisson_stream_completes(torch_cuda):
    from phasefield5d_b200.serving import poisson_arrivals
    reqs = _requests(steps=80)
    srv, st = _serve(reqs, poisson_arrivals(30.0, len(reqs), seed=4))
    assert st["requests_done"] == len(reqs)
    assert 0 < st["p50_time_to_solution_s"] <= st["p99_time_to_solution_s"]
    assert st["grid_point_steps_per_s"] > 0


def test_fp64_backend_alone_equals_mix(torch_cuda):
    """The plain-FP64 comparison backend (one FP64 stepper per request):
    every request's result is bit-identical alone and in the mix."""
    import copy
    reqs = _requests(steps=60)[:4]
    srv, st = _serve([copy.copy(r) for r in reqs], [0.0, 0.01, 0.02, 0.03], precision="fp64")
    assert st["requests_done"] == len(reqs)
    mixed = {r.rid: r for r in srv.finished}
    for r in reqs:
        alone_srv, _st = _serve([copy.copy(r)], [0.0], precision="fp64")
        alone = alone_srv.finished[0]
        assert alone.final_state["step"] == mixed[r.rid].final_state["step"] == r.n_steps
        assert np.array_equal(alone.result, mixed[r.rid].result), r.rid


def test_halting_and_cancelled_requests_leave_others_intact(torch_cuda):
    """A request whose field is bad from the start halts at its first
    out-of-bounds check and retires; another is cancelled while active.  The
    remaining requests finish with the results they have alone."""
    import copy
    from phasefield5d_b200.serving import Server
    reqs = _requests(steps=60)[:4]              # 1D, 2D, 3D, 1D
    bad = copy.copy(reqs[1])
    prob = copy.copy(bad.problem)
    X = prob.X_init.copy()
    X[2, 3, 1] = np.nan
    prob.X_init = X
    bad.problem = prob
    reqs[1] = bad
    srv = Server(step_block=10, reserve_bytes=0)
    for r, a in zip([copy.copy(r) for r in reqs], [0.0, 0.0, 0.0, 0.0]):
        r.arrival = a
        srv.submit(r)
    for _ in range(3):
        srv.tick()
    assert srv.cancel(reqs[2].rid)               # the 3D request, while active
    srv.run(timeout=300)
    status = {r.rid: r.status for r in srv.finished}
    assert status == {0: "done", 1: "halted", 2: "cancelled", 3: "done"}
    for rid in (0, 3):
        alone_srv, _ = _serve([copy.copy(reqs[rid])], [0.0])
        mixed = next(r for r in srv.finished if r.rid == rid)
        assert np.array_equal(alone_srv.finished[0].result, mixed.result), rid
