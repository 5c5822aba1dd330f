"""Fixture for the full-length plain FP64 parity test: the oracle (bit-for-bit
the reference's kernels, pinned by make_golden.py) runs the 2D 512x512
adaptive workload for all of its 20,000 steps on the CPU; the final field is
stored at 4096 seeded sample points together with per-component sums,
minima and maxima, and the final time / dt / max |dX/dt|.

    python tests/golden/make_fullrun.py          # ~10-30 min on 8-16 host threads
"""
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)

from oracle.oracle import OracleStepper  # noqa: E402
from phasefield5d_b200 import workload as W  # noqa: E402

N_SAMPLES = 4096


def main():
    cfg = W.config_2d_adaptive()
    prob = W.build_problem(cfg)
    n = cfg.total_timesteps
    st = OracleStepper.from_problem(prob, fft_workers=-1)
    t0 = time.time()
    ok = st.run(n)
    X = st.X.reshape(-1, 4)
    rng = np.random.default_rng(20000)
    idx = np.sort(rng.choice(X.shape[0], size=N_SAMPLES, replace=False))
    np.savez_compressed(os.path.join(HERE, "full2d_20k.npz"), steps=np.int64(st.step_index),
                        completed=np.bool_(ok), idx=idx, X=X[idx], sums=X.sum(axis=0),
                        mins=X.min(axis=0), maxs=X.max(axis=0), time=np.float64(st.time),
                        dt=np.float64(st.dt), xdotmax=np.float64(st.xdotmax),
                        omega_seed=np.int64(prob.omega_seed))
    print(f"{n} oracle steps in {time.time() - t0:.0f} s; fixture written")


if __name__ == "__main__":
    main()
