"""The 1D elastic term's closed form, on the host.

A 1D solve's B(k) depends on k only through its sign, so it is one value bn
for every k != 0 and b0 at k = 0.  Then irfft(B * rfft(s)) equals
bn * (s - mean s) + b0 * mean s exactly, which is what the steppers evaluate
in one kernel for 1D solves up to 16384 points (they check the flatness of
B(k) exactly at creation and keep the FFT path otherwise).  These tests pin
the precondition on the library's own B(k) and the identity itself.
"""
import numpy as np


def test_1d_bk_is_flat_away_from_k0():
    from phasefield5d_b200 import workload as W
    prob = W.build_problem(W.config_1d_fixed())
    bk = np.asarray(prob.bk)
    assert bk.shape == (prob.shape[0] // 2 + 1,)
    assert np.all(bk[1:] == bk[1])          # exactly, as the steppers test it


def test_closed_form_equals_fft_path():
    rng = np.random.default_rng(7)
    for n in (1280, 1281, 64):
        s = rng.standard_normal(n) * 1e-3
        bn, b0 = -2.0954982e11, 0.0
        bk = np.full(n // 2 + 1, bn)
        bk[0] = b0
        via_fft = np.fft.irfft(bk * np.fft.rfft(s), n=n)
        mean = s.sum() / n
        closed = bn * (s - mean) + b0 * mean
        assert np.max(np.abs(via_fft - closed)) <= 1e-12 * np.max(np.abs(closed))
        b0 = 3.0e10                          # a non-zero k = 0 value too
        bk[0] = b0
        via_fft = np.fft.irfft(bk * np.fft.rfft(s), n=n)
        closed = bn * (s - mean) + b0 * mean
        assert np.max(np.abs(via_fft - closed)) <= 1e-12 * np.max(np.abs(closed))
