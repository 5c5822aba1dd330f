"""GPU parity of the fused FP64 step loop.

* Small 1D/2D/3D trajectories against the reference's own golden runs
  (tests/golden/trajectories.npz).
* The plain-FP64 workloads at full size against the CPU oracle: 1D 1280 for
  the full 10,000 fixed-dt steps, 2D 512x512 adaptive for a prefix of
  steps, 3D on odd shapes.
* Properties at full size: mass conservation over 20,000 2D steps, graph
  block boundaries invisible, out-of-bounds halts.

Tolerance (plain FP64): max |X_gpu - X_ref| <= 1e-12 * max |X_ref| after N
steps.  The only non-bitwise step is the FFT (cuFFT vs pocketfft); the
stricter X - X0 deviation is reported in the assertion messages.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FIELD_RTOL = 1e-12


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _rel(got, want, X0):
    a = float(np.max(np.abs(got - want)))
    return a / float(np.max(np.abs(want))), a / max(float(np.max(np.abs(want - X0))), 1e-300)


def _golden_stepper(g, name, small_table):
    from phasefield5d_b200.solver.table import node_coordinates
    from phasefield5d_b200.stepper import Stepper
    sc = g[f"{name}_scalars"]
    dx, ctld, t_cfl, dt_nom, kappa_value, adaptive, n = sc[:7]
    adaptive = bool(adaptive)
    dt0 = dt_nom if adaptive else min(dt_nom, 0.005 * ctld, t_cfl)
    st = Stepper(grid=small_table["grid"], resolution=small_table["resolution"],
                 node_coord=node_coordinates(small_table["tree"], small_table["resolution"]),
                 X=g[f"{name}_X_init"], X0=g[f"{name}_X0"], kappa=np.full(4, kappa_value), dx=dx,
                 lvec=g[f"{name}_lvec"], bk=g[f"{name}_bk"], ctld=ctld, t_cfl=t_cfl, dt=dt0,
                 adaptive=adaptive, lower_limit=sc[7], upper_limit=sc[8])
    return st, int(n)


@pytest.mark.parametrize("name", ["1d_fixed", "1d_adapt", "2d_adapt", "3d_adapt"])
def test_golden_trajectory(torch_cuda, small_table, traj_golden, name):
    g = traj_golden
    st, n = _golden_stepper(g, name, small_table)
    state = st.run(n)
    X = st.X.cpu().numpy()
    want = g[f"{name}_X_final"]
    r_field, r_dev = _rel(X, want, g[f"{name}_X0"])
    assert state["step"] == n and not state["halted"]
    assert r_field <= FIELD_RTOL, f"{name}: field rel {r_field:.2e} (X-X0 rel {r_dev:.2e})"
    assert abs(state["time"] - float(g[f"{name}_time"])) <= 1e-12 * float(g[f"{name}_time"])
    assert abs(state["dt"] - g[f"{name}_dts"][-1]) <= 1e-12 * g[f"{name}_dts"][-1]
    st.close()


def _problem(mk, **over):
    from phasefield5d_b200 import workload as W
    cfg = mk()
    for k, v in over.items():
        setattr(cfg, k, v)
    return W.build_problem(cfg)


def test_1d_full_fixed_dt_vs_oracle(torch_cuda):
    """1D 1280 cells, fixed dt, all 10,000 steps."""
    from oracle.oracle import OracleStepper
    from phasefield5d_b200 import workload as W
    from phasefield5d_b200.stepper import Stepper
    prob = _problem(W.config_1d_fixed)
    n = prob.cfg.total_timesteps
    gpu = Stepper.from_problem(prob)
    state = gpu.run(n)
    ref = OracleStepper.from_problem(prob)
    ref.run(n)
    r_field, r_dev = _rel(gpu.X.cpu().numpy(), ref.X, prob.X0)
    assert state["step"] == n
    assert r_field <= FIELD_RTOL, f"field rel {r_field:.2e} (X-X0 rel {r_dev:.2e})"
    assert state["time"] == pytest.approx(ref.time, rel=1e-14)
    gpu.close()


def test_2d_512_adaptive_prefix_vs_oracle(torch_cuda):
    """2D 512x512 adaptive: the first 200 steps against the oracle."""
    from oracle.oracle import OracleStepper
    from phasefield5d_b200 import workload as W
    from phasefield5d_b200.stepper import Stepper
    prob = _problem(W.config_2d_adaptive)
    n = 200
    gpu = Stepper.from_problem(prob)
    state = gpu.run(n)
    ref = OracleStepper.from_problem(prob)
    ref.run(n)
    r_field, r_dev = _rel(gpu.X.cpu().numpy(), ref.X, prob.X0)
    assert r_field <= FIELD_RTOL, f"field rel {r_field:.2e} (X-X0 rel {r_dev:.2e})"
    assert state["dt"] == pytest.approx(ref.dt, rel=1e-12)
    assert state["xdotmax"] == pytest.approx(ref.xdotmax, rel=1e-10)
    gpu.close()


def test_2d_512_full_20k_vs_oracle_fixture(torch_cuda):
    """All 20,000 adaptive steps of the 2D 512x512 workload against the
    oracle's run of the same steps (tests/golden/full2d_20k.npz, written by
    tests/golden/make_fullrun.py): the field at 4096 sample points and the
    per-component minima / maxima within 1e-12 of max|X|, the per-component
    sums and the final clock within 1e-12 relative."""
    import os
    from phasefield5d_b200 import workload as W
    from phasefield5d_b200.stepper import Stepper
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "full2d_20k.npz"))
    prob = _problem(W.config_2d_adaptive)
    assert prob.omega_seed == int(g["omega_seed"]) and bool(g["completed"])
    gpu = Stepper.from_problem(prob)
    state = gpu.run(int(g["steps"]))
    X = gpu.X.cpu().numpy().reshape(-1, 4)
    gpu.close()
    scale = float(np.max(np.abs(g["maxs"])))
    assert state["step"] == int(g["steps"]) and not state["halted"]
    err = np.max(np.abs(X[g["idx"]] - g["X"]))
    assert err <= FIELD_RTOL * scale, f"sampled field err {err:.2e}"
    assert np.all(np.abs(X.min(axis=0) - g["mins"]) <= FIELD_RTOL * scale)
    assert np.all(np.abs(X.max(axis=0) - g["maxs"]) <= FIELD_RTOL * scale)
    assert np.all(np.abs(X.sum(axis=0) - g["sums"]) <= FIELD_RTOL * np.abs(g["sums"]))
    assert state["time"] == pytest.approx(float(g["time"]), rel=1e-12)
    assert state["dt"] == pytest.approx(float(g["dt"]), rel=1e-10)


def test_2d_512_full_run_conserves_mass(torch_cuda):
    """All 20,000 adaptive steps on the GPU: the flux form conserves each
    component's mean (up to rounding), no halt, finite field."""
    from phasefield5d_b200 import workload as W
    from phasefield5d_b200.stepper import Stepper
    prob = _problem(W.config_2d_adaptive)
    gpu = Stepper.from_problem(prob)
    m0 = prob.X_init.reshape(-1, 4).mean(axis=0)
    state = gpu.run(prob.cfg.total_timesteps)
    X = gpu.X.cpu().numpy()
    assert state["step"] == prob.cfg.total_timesteps and not state["halted"]
    assert np.isfinite(X).all()
    drift = np.max(np.abs(X.reshape(-1, 4).mean(axis=0) - m0))
    assert drift <= 1e-13, drift
    gpu.close()


@pytest.mark.parametrize("shape,n", [((20, 18, 24), 12), ((10, 13, 37), 8), ((7, 33), 40),
                                     ((131,), 60)])
def test_odd_shapes_vs_oracle(torch_cuda, shape, n):
    """Shapes that are not multiples of the tiles (partial tiles, wrap-around halos)."""
    from oracle.oracle import OracleStepper
    from phasefield5d_b200 import workload as W
    from phasefield5d_b200.stepper import Stepper
    cfg = W.SolveConfig(system_dim=len(shape), initial_composition=(0.1, 0.2, 0.2, 0.25),
                        resolution=0.05, kappa_value=5e-16, mw=4, ppw=16, shape=shape,
                        adaptive=True, n_k=2000, fluctuation=3e-2)
    prob = W.build_problem(cfg)
    gpu = Stepper.from_problem(prob)
    gpu.run(n)
    ref = OracleStepper.from_problem(prob)
    ref.run(n)
    r_field, r_dev = _rel(gpu.X.cpu().numpy(), ref.X, prob.X0)
    assert r_field <= FIELD_RTOL, f"{shape}: field rel {r_field:.2e} (X-X0 rel {r_dev:.2e})"
    gpu.close()


@pytest.mark.parametrize("shape", [(8, 30), (16, 24), (32, 40), (64, 22), (128, 18), (256, 10),
                                   (1024, 6)])
def test_column_pass_lengths_vs_oracle(torch_cuda, shape):
    """2D fields whose axis 0 is a power of two run the elastic term through
    cuFFT's row transforms and the column kernel (mixed-radix transform
    along axis 0, B(k)/N, inverse): every transform length from 8 to 1024
    (radix-8 stages with a radix-4 or radix-2 tail) against the oracle's
    pocketfft path, 25 steps at the parity tolerance."""
    from oracle.oracle import OracleStepper
    from phasefield5d_b200 import workload as W
    from phasefield5d_b200.stepper import Stepper
    cfg = W.SolveConfig(system_dim=2, initial_composition=(0.1, 0.2, 0.2, 0.25), resolution=0.05,
                        kappa_value=5e-16, mw=4, ppw=16, shape=shape, adaptive=True, n_k=2000,
                        fluctuation=3e-2)
    prob = W.build_problem(cfg)
    gpu = Stepper.from_problem(prob)
    gpu.run(25)
    ref = OracleStepper.from_problem(prob)
    ref.run(25)
    r_field, r_dev = _rel(gpu.X.cpu().numpy(), ref.X, prob.X0)
    assert r_field <= FIELD_RTOL, f"{shape}: field rel {r_field:.2e} (X-X0 rel {r_dev:.2e})"
    gpu.close()


def test_nearest_row_fallback_inside_step(torch_cuda):
    """Composition straddling the linear-region threshold: part of the field
    takes the nearest-row branch every step."""
    from oracle.oracle import OracleStepper
    from phasefield5d_b200 import workload as W
    from phasefield5d_b200.stepper import Stepper
    cfg = W.SolveConfig(system_dim=2, initial_composition=(0.1, 0.2, 0.2, 0.25), resolution=0.05,
                        kappa_value=5e-16, mw=4, ppw=16, shape=(24, 20), adaptive=True, n_k=2000)
    prob = W.build_problem(cfg)
    rng = np.random.default_rng(11)
    X = prob.X_init.copy()
    X[..., 3] += rng.uniform(0.0, 0.1, size=X.shape[:-1])      # sums up to 0.85 > 0.8 threshold
    prob.X_init = X
    gpu = Stepper.from_problem(prob)
    state = gpu.run(30)
    ref = OracleStepper.from_problem(prob)
    ref.run(30)
    assert state["flags"] & 0x20            # nearest-row branch used
    r_field, _ = _rel(gpu.X.cpu().numpy(), ref.X, prob.X0)
    assert r_field <= FIELD_RTOL
    gpu.close()


def test_graph_blocks_are_invisible(torch_cuda):
    """advance(37) + advance(83) equals advance(120) bit for bit."""
    from phasefield5d_b200 import workload as W
    from phasefield5d_b200.stepper import Stepper
    cfg = W.SolveConfig(system_dim=2, initial_composition=(0.1, 0.2, 0.2, 0.25), resolution=0.05,
                        kappa_value=5e-16, mw=4, ppw=16, shape=(40, 36), adaptive=True, n_k=2000)
    prob = W.build_problem(cfg)
    a = Stepper.from_problem(prob)
    a.advance(37)
    a.advance(83)
    sa = a.state()
    b = Stepper.from_problem(prob)
    sb = b.run(120)
    assert sa == sb
    assert np.array_equal(a.X.cpu().numpy(), b.X.cpu().numpy())
    a.close()
    b.close()


@pytest.mark.parametrize("inject", ["nan", "sum_over_one", "negative"])
def test_out_of_bounds_halts(torch_cuda, inject):
    """Host-made failure: a bad initial field halts the loop at the step-0
    check (simulate.py:231) with the field untouched."""
    from phasefield5d_b200 import workload as W
    from phasefield5d_b200.stepper import Stepper
    cfg = W.SolveConfig(system_dim=1, initial_composition=(0.1, 0.2, 0.2, 0.25), resolution=0.05,
                        kappa_value=5e-16, mw=4, ppw=16, shape=(64,), adaptive=True, n_k=2000)
    prob = W.build_problem(cfg)
    X = prob.X_init.copy()
    if inject == "nan":
        X[5, 2] = np.nan
    elif inject == "sum_over_one":
        X[7] = [0.3, 0.3, 0.3, 0.2]
    else:
        X[9, 1] = -0.01
    prob.X_init = X
    gpu = Stepper.from_problem(prob)
    state = gpu.run(50)
    assert state["halted"] and state["step"] == 0 and state["time"] == 0.0
    got = gpu.X.cpu().numpy()
    assert np.array_equal(np.isnan(got), np.isnan(X))
    assert np.array_equal(np.nan_to_num(got), np.nan_to_num(X))
    gpu.close()


@pytest.mark.parametrize("dim,shape", [(1, (64,)), (2, (40, 36)), (3, (12, 20, 24))])
def test_nonfinite_midrun_raises_like_reference(torch_cuda, dim, shape):
    """Host-made failure between steps: a NaN written into the field after 5
    steps reaches the nearest-row fallback at the next step (NaN fails the
    linear-region test), where the reference's cKDTree.query raises
    ValueError.  The stepper halts before that step's update and ``run``
    raises ValueError; the field and the step count stay as they were."""
    from oracle.oracle import OracleStepper
    from phasefield5d_b200 import workload as W
    from phasefield5d_b200.stepper import Stepper
    cfg = W.SolveConfig(system_dim=dim, initial_composition=(0.1, 0.2, 0.2, 0.25),
                        resolution=0.05, kappa_value=5e-16, mw=4, ppw=16, shape=shape,
                        adaptive=True, n_k=2000)
    prob = W.build_problem(cfg)
    gpu = Stepper.from_problem(prob)
    gpu.run(5)
    bad = (0,) * (dim - 1) + (3,)
    gpu.X[bad + (1,)] = float("nan")
    before = gpu.X.cpu().numpy()
    with pytest.raises(ValueError):
        gpu.run(10)
    st = gpu.state()
    assert st["halted"] and st["nn_nonfinite"] and st["step"] == 5
    after = gpu.X.cpu().numpy()
    assert np.array_equal(after, before, equal_nan=True)
    ref = OracleStepper.from_problem(prob)
    ref.run(5)
    ref.X[bad + (1,)] = np.nan
    with pytest.raises(ValueError):
        ref.step()
    gpu.close()


@pytest.mark.parametrize("precision", ["fp64", "fp32c"])
def test_near_face_point_takes_row_inside_step(torch_cuda, precision):
    """A point near the simplex face (row sum 0.99, past the 0.8 linear
    threshold of the 0.05 table) takes the nearest table row inside the
    fused step, in both forms, with the fallback reported and no error
    flag; the FP64 form still tracks the oracle."""
    from oracle.oracle import OracleStepper
    from phasefield5d_b200 import workload as W
    from phasefield5d_b200.stepper import Stepper
    cfg = W.SolveConfig(system_dim=2, initial_composition=(0.1, 0.2, 0.2, 0.25), resolution=0.05,
                        kappa_value=5e-16, mw=4, ppw=16, shape=(24, 20), adaptive=True, n_k=2000)
    prob = W.build_problem(cfg)
    X = prob.X_init.copy()
    X[3, 4] = [0.28, 0.25, 0.24, 0.22]
    prob.X_init = X
    gpu = Stepper.from_problem(prob, precision=precision)
    st = gpu.run(3)
    assert st["nn_used"] and not (st["nn_far"] or st["nn_nonfinite"] or st["nn_no_row"])
    if precision == "fp64":
        ref = OracleStepper.from_problem(prob)
        ref.run(3)
        r_field, _ = _rel(gpu.X.cpu().numpy(), ref.X, prob.X0)
        assert r_field <= FIELD_RTOL
    gpu.close()


def test_rate_variants_bitwise_identical(torch_cuda):
    """Every autotuner variant (tile shape x occupancy) computes each point
    the same way, so trajectories are bit-identical across variants."""
    from phasefield5d_b200 import workload as W
    from phasefield5d_b200.stepper import Stepper
    for dim, shape in [(2, (40, 70)), (3, (12, 20, 36))]:
        cfg = W.SolveConfig(system_dim=dim, initial_composition=(0.1, 0.2, 0.2, 0.25),
                            resolution=0.05, kappa_value=5e-16, mw=4, ppw=16, shape=shape,
                            adaptive=True, n_k=2000, fluctuation=2e-2)
        prob = W.build_problem(cfg)
        ref = None
        st0 = Stepper.from_problem(prob, autotune=False)
        n_variants = st0.n_variants
        st0.close()
        for v in range(n_variants):
            st = Stepper.from_problem(prob, autotune=False)
            st.set_variant(v)
            st.run(7)
            X = st.X.cpu().numpy()
            st.close()
            if ref is None:
                ref = X
            assert np.array_equal(X, ref), (dim, v)
