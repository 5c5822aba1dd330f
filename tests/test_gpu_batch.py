"""Batched form (many FP32-compensated 1D/2D solves per launch).

* Each solve of a batch tracks its own plain-FP64 single-solve run within
  the precision tolerance (max |X_batch - X_fp64| <= 1e-6 * max |X_fp64|).
* A solve gives the same result alone and inside a mixed batch: bit for bit
  for 1D solves (no FFT); within 1e-6 for 2D solves (cuFFT may pick another
  algorithm for a different plan batch count).
* A solve that halts on a bad field leaves the other solves untouched.
"""
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


def _small_batch():
    from phasefield5d_b200 import workload as W
    cfgs = W.batched_configs(8, seed=5, steps=300)
    shapes = [(512,), (40, 36), (700,), (64, 64), (1030,), (48, 80), (256,), (32, 32)]
    for c, sh in zip(cfgs, shapes):
        c.shape = sh
        c.system_dim = len(sh)
    probs, _ = W.build_batched_problems(cfgs)
    return probs


@pytest.fixture(scope="module")
def small_probs(torch_cuda):
    return _small_batch()


def _fp64(prob, n):
    from phasefield5d_b200.stepper import Stepper
    st = Stepper.from_problem(prob, precision="fp64")
    st.run(n)
    X = st.X.cpu().numpy()
    st.close()
    return X


def test_batch_tracks_fp64(small_probs):
    from phasefield5d_b200.batch import BatchStepper
    n = 300
    b = BatchStepper(small_probs)
    b.advance(n)
    states = b.states()
    for i, p in enumerate(small_probs):
        assert states[i]["step"] == n and not states[i]["halted"], (i, states[i])
        Xb = b.field(i).cpu().numpy()
        X64 = _fp64(p, n)
        err = np.max(np.abs(Xb - X64)) / np.max(np.abs(X64))
        assert err <= FIELD_RTOL_FP32C, (i, p.shape, err)
    b.close()


def test_workload_sized_solves_track_fp64(torch_cuda):
    """2D solves at the batched workload's sizes (squares 128^2 to 368^2,
    prime factors 3, 23 in the FFT lengths) beside a small non-square one:
    each tracks its plain-FP64 run within the precision tolerance."""
    from phasefield5d_b200 import workload as W
    from phasefield5d_b200.batch import BatchStepper
    cfgs = W.batched_configs(4, seed=9, steps=200)
    for c, sh in zip(cfgs, [(128, 128), (144, 144), (48, 40), (368, 368)]):
        c.shape = sh
        c.system_dim = 2
    probs, _ = W.build_batched_problems(cfgs)
    n = 200
    b = BatchStepper(probs)
    b.advance(n)
    for i, p in enumerate(probs):
        Xb = b.field(i).cpu().numpy()
        X64 = _fp64(p, n)
        err = np.max(np.abs(Xb - X64)) / np.max(np.abs(X64))
        assert err <= FIELD_RTOL_FP32C, (i, p.shape, err)
    b.close()


def test_alone_vs_mix(small_probs):
    from phasefield5d_b200.batch import BatchStepper
    n = 120
    mix = BatchStepper(small_probs, autotune=False)
    mix.advance(n)
    for i, p in enumerate(small_probs):
        alone = BatchStepper([p], autotune=False)
        alone.advance(n)
        a = alone.field(0).cpu().numpy()
        m = mix.field(i).cpu().numpy()
        assert alone.states()[0]["time"] == mix.states()[i]["time"] or p.dim == 2
        if p.dim == 1:
            assert np.array_equal(a, m), i
        else:
            assert np.max(np.abs(a - m)) <= FIELD_RTOL_FP32C * np.max(np.abs(m)), i
        alone.close()
    mix.close()


def test_variants_agree(small_probs):
    """Every batch-kernel variant computes each point the same way."""
    from phasefield5d_b200.batch import BatchStepper
    ref = None
    from phasefield5d_b200 import _lib
    for v in range(int(_lib.load().pf5d_batch_variant_count())):
        b = BatchStepper(small_probs[:4], autotune=False)
        b.set_variant(v)
        b.advance(9)
        fields = [b.field(i).cpu().numpy() for i in range(4)]
        b.close()
        if ref is None:
            ref = fields
        for f, r in zip(fields, ref):
            assert np.array_equal(f, r), v


def test_halted_solve_isolated(small_probs):
    import copy
    from phasefield5d_b200.batch import BatchStepper
    probs = [copy.copy(p) for p in small_probs[:4]]
    X = probs[1].X_init.copy()
    X[3, 5, 2] = np.nan
    probs[1].X_init = X
    n = 60
    b = BatchStepper(probs, autotune=False)
    b.advance(n)
    st = b.states()
    assert st[1]["halted"] and st[1]["step"] == 0
    ref = BatchStepper([p for k, p in enumerate(probs) if k != 1], autotune=False)
    ref.advance(n)
    for k_mix, k_ref in [(0, 0), (2, 1), (3, 2)]:
        assert st[k_mix]["step"] == n and not st[k_mix]["halted"]
        a = b.field(k_mix).cpu().numpy()
        r = ref.field(k_ref).cpu().numpy()
        if probs[k_mix].dim == 1:
            assert np.array_equal(a, r)
        else:
            assert np.max(np.abs(a - r)) <= FIELD_RTOL_FP32C * np.max(np.abs(r))
    b.close()
    ref.close()


def test_full_batched_workload_short_run(torch_cuda):
    """The 64-solve batched workload (uneven 1D 2048-8192 / 2D 128^2-384^2,
    four temperature tables): 200 steps, no halt, finite, spot-checked
    against FP64 single-solve runs."""
    from phasefield5d_b200 import workload as W
    from phasefield5d_b200.batch import BatchStepper
    probs, _ = W.build_batched_problems(W.batched_configs(64))
    b = BatchStepper(probs)
    n = 200
    b.advance(n)
    st = b.states()
    assert all(s["step"] == n and not s["halted"] for s in st)
    for i in (0, 1, 31, 62):
        Xb = b.field(i).cpu().numpy()
        assert np.isfinite(Xb).all()
        X64 = _fp64(probs[i], n)
        assert np.max(np.abs(Xb - X64)) <= FIELD_RTOL_FP32C * np.max(np.abs(X64)), i
    b.close()
