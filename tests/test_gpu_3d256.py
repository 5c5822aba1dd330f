"""The 3D 256^3 workload (51^4 table, elasticity on, adaptive dt) at full size.

This is the one named workload whose field (537 MB in FP64, 268 MB per FP32
half) is larger than the B200's L2, so its kernels run from HBM.

* Plain FP64 against the CPU oracle for a 3-step prefix: max |X_gpu - X_ref|
  <= 1e-12 * max |X_ref| (the only non-bitwise step is cuFFT vs pocketfft),
  with the clock and dt held to 1e-12.
* FP32-compensated against plain FP64 on the GPU for 500 steps: max |X_fp32c
  - X_fp64| <= 1e-6 * max |X_fp64|, mass drift of the mean composition
  <= 1e-12, matching clocks.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FIELD_RTOL = 1e-12
FIELD_RTOL_FP32C = 1e-6
MASS_DRIFT_TOL = 1e-12


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


@pytest.fixture(scope="module")
def prob3d():
    from phasefield5d_b200 import workload as W
    return W.build_problem(W.config_3d_precision())


def test_3d_256_fp64_prefix_vs_oracle(torch_cuda, prob3d):
    from oracle.oracle import OracleStepper
    from phasefield5d_b200.stepper import Stepper
    prob = prob3d
    assert prob.shape == (256, 256, 256) and prob.grid.shape[0] == 51
    n = 3
    gpu = Stepper.from_problem(prob)
    state = gpu.run(n)
    X = gpu.X.cpu().numpy()
    gpu.close()
    ref = OracleStepper.from_problem(prob)
    ref.run(n)
    scale = float(np.max(np.abs(ref.X)))
    err = float(np.max(np.abs(X - ref.X)))
    dev = float(np.max(np.abs(ref.X - prob.X0)))
    assert state["step"] == n and not state["halted"]
    assert err <= FIELD_RTOL * scale, f"field rel {err / scale:.2e} (X-X0 rel {err / dev:.2e})"
    assert state["time"] == pytest.approx(ref.time, rel=1e-12)
    assert state["dt"] == pytest.approx(ref.dt, rel=1e-12)


def test_3d_256_fp32c_vs_fp64_500_steps(torch_cuda, prob3d):
    from phasefield5d_b200.precision import compare_forms
    rep = compare_forms(prob3d, 500)
    assert not rep["halted"], rep
    assert rep["max_rel_err_X"] <= FIELD_RTOL_FP32C, rep
    assert max(abs(v) for v in rep["mass_drift_fp32c"]) <= MASS_DRIFT_TOL, rep
    assert rep["time_fp32c"] == pytest.approx(rep["time_fp64"], rel=1e-6), rep
