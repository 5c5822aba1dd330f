"""Save-step diagnostics on the GPU (pf5d_stepper_step_save) against the
oracle's restatement of examples/simulate.py:299-354, and the device driver
against the oracle's main loop (same save steps, same files and traces).

Tolerances: values that are sums or reductions of the field take the FFT
rounding difference of the plain FP64 path (1e-12 relative on the fields)
plus a different summation order; the total flux and the net change are
rounding noise around zero, compared on the scale of the summed |terms|."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

RTOL = 1e-10


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _problem(dim, shape):
    from phasefield5d_b200 import workload as W
    cfg = W.SolveConfig(system_dim=dim, initial_composition=(0.1, 0.2, 0.2, 0.25),
                        resolution=0.05, kappa_value=5e-16, mw=4, ppw=16, shape=shape,
                        adaptive=True, n_k=2000, fluctuation=2e-2)
    return W.build_problem(cfg)


def _close(a, b, scale, rtol=RTOL):
    a, b = np.asarray(a, dtype=float), np.asarray(b, dtype=float)
    return np.all(np.abs(a - b) <= rtol * scale)


@pytest.mark.parametrize("dim,shape", [(1, (96,)), (2, (24, 20)), (3, (8, 10, 12))])
def test_step_save_matches_oracle(torch_cuda, dim, shape):
    from oracle.oracle import OracleStepper
    from phasefield5d_b200.stepper import Stepper
    prob = _problem(dim, shape)
    st = Stepper.from_problem(prob)
    ost = OracleStepper.from_problem(prob)
    for k in range(4):
        g = st.step_save()
        r = ost.step_save()
        assert not g["halted"] and g["step"] == r["step"] == k
        for key in ("dt", "time", "xdotmax"):
            assert _close(g[key], r[key], abs(r[key])), (key, g[key], r[key])
        for key in ("mass", "comp_min", "comp_max", "max_change"):
            assert _close(g[key], r[key], np.abs(r[key])), (key, g[key], r[key])
        assert _close(g["comp_fe_min"], r["comp_fe_min"], 1.0)
        assert _close(g["comp_var"], r["comp_var"], np.abs(r["comp_var"]), 1e-8), \
            (g["comp_var"], r["comp_var"])
        assert _close(g["f_grad"], r["f_grad"], abs(r["f_grad"]), 1e-8)
        n = int(np.prod(shape))
        assert _close(g["net"], r["net"], n * r["xdotmax"], 1e-12), (g["net"], r["net"])
        assert _close(g["total_flux"], r["total_flux"], r["flux_abs"], 1e-12)
    X = st.X.cpu().numpy()
    assert np.max(np.abs(X - ost.X)) <= 1e-12 * np.max(np.abs(ost.X))
    st.close()


def test_driver_matches_oracle_loop(torch_cuda, tmp_path):
    """Same save steps, state files and trace rows as the oracle's
    step-by-step main loop; most steps run as graph blocks."""
    from oracle.oracle import OracleStepper, run_simulation as oracle_run
    from phasefield5d_b200.driver import run_simulation
    from phasefield5d_b200.stepper import Stepper
    prob = _problem(2, (24, 20))
    # about one data save every 20 steps at the capped dt
    frames = max(1, int(prob.ctld / (20.0 * min(prob.t_cfl, 0.005 * prob.ctld))))
    kw = dict(ctld=prob.ctld, t_cfl=prob.t_cfl, early_stage_frames=frames,
              late_burst_duration_ctld=2, late_burst_frames=30, late_tail_frames=1)
    n = 400
    st = Stepper.from_problem(prob)
    tg, fg = run_simulation(st, n, str(tmp_path / "gpu"), **kw)
    tr, fr = oracle_run(OracleStepper.from_problem(prob), n, str(tmp_path / "ref"), **kw)
    assert tg["timestep"] == tr["timestep"] and len(tg["timestep"]) > 3
    assert [p.split("/")[-1] for p in fg] == [p.split("/")[-1] for p in fr]
    for a, b in zip(fg, fr):
        za, zb = np.load(a), np.load(b)
        assert int(za["timestep"]) == int(zb["timestep"])
        assert abs(float(za["time"]) - float(zb["time"])) <= 1e-12 * abs(float(zb["time"]))
        Xa, Xb = za["current_composition"], zb["current_composition"]
        assert Xa.shape == Xb.shape and Xa.dtype == Xb.dtype
        assert np.max(np.abs(Xa - Xb)) <= 1e-12 * np.max(np.abs(Xb))
    for key in ("time", "dt", "composition_change_max", "comp_fe_min"):
        a, b = np.array(tg[key]), np.array(tr[key])
        assert np.all(np.abs(a - b) <= RTOL * np.abs(b) + 1e-300), key
    st.close()


@pytest.mark.parametrize("dim,shape", [(1, (96,)), (2, (24, 20)), (3, (8, 10, 12))])
def test_step_save_fp32c_tracks_fp64(torch_cuda, dim, shape):
    """The precision form's save-step diagnostics follow the FP64 form's
    within the FP32c field tolerance (1e-6 relative) on the same steps."""
    from phasefield5d_b200.stepper import Stepper
    prob = _problem(dim, shape)
    a = Stepper.from_problem(prob)
    b = Stepper.from_problem(prob, precision="fp32c")
    for k in range(3):
        g = a.step_save()
        f = b.step_save()
        assert g["step"] == f["step"] == k and not f["halted"]
        for key in ("mass", "comp_min", "comp_max", "max_change"):
            assert _close(f[key], g[key], np.abs(g[key]), 1e-5), (key, f[key], g[key])
        assert _close(f["comp_fe_min"], g["comp_fe_min"], 1.0, 1e-6)
        assert _close(f["dt"], g["dt"], abs(g["dt"]), 1e-6)
        assert np.all(np.isfinite(f["total_flux"])) and np.isfinite(f["f_grad"])
    a.close()
    b.close()
