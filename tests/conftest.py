"""Shared test fixtures.

Tests marked ``gpu`` need a CUDA device and the built CUDA library; all other
tests run on the CPU (oracle vs golden vectors, host logic, C-ABI symbol
checks, gloo multi-process tests).
"""
import os
import sys

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(REPO, "tests", "golden")
if REPO not in sys.path:
    sys.path.insert(0, REPO)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device and the built CUDA library")


@pytest.fixture(scope="session")
def golden_dir():
    return GOLDEN


@pytest.fixture(scope="session")
def small_table():
    """The 0.05-spacing synthetic table used by the small golden cases:
    (data rows, dense grid, KD-tree, row values, resolution)."""
    from phasefield5d_b200.solver.table import build_4d_grid, build_calphad_kdtree
    z = np.load(os.path.join(GOLDEN, "table_small.npz"))
    data = z["data"]
    res = float(z["resolution"])
    _, grid = build_4d_grid(data, res)
    tree, vals = build_calphad_kdtree(data)
    return dict(data=data, grid=grid, tree=tree, vals=vals, resolution=res)


@pytest.fixture(scope="session")
def kernels_golden():
    return dict(np.load(os.path.join(GOLDEN, "kernels.npz")))


@pytest.fixture(scope="session")
def traj_golden():
    return dict(np.load(os.path.join(GOLDEN, "trajectories.npz")))


def cuda_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False
