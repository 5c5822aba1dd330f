"""C-ABI checks that need no GPU: libpf5d.so loads, exports every entry
point include/pf5d.h declares, and its host-side adaptive-dt rule matches the
reference's golden cases."""
import os
import re
import subprocess

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(REPO, "include", "pf5d.h")


def declared_symbols():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(pf5d_[a-z0-9_]+)\s*\(", src)))


@pytest.fixture(scope="module")
def lib():
    from phasefield5d_b200 import _lib
    if not os.path.exists(_lib.LIB_PATH):
        subprocess.run(["make", "-s", "-C", os.path.join(REPO, "phasefield5d_b200", "csrc")],
                       check=True)
    return _lib.load(require_cuda=False)


def test_header_declares_expected_surface():
    syms = declared_symbols()
    for name in ["pf5d_interp4d", "pf5d_laplacian", "pf5d_divergence_from_mu", "pf5d_abs_max",
                 "pf5d_clamp_simplex", "pf5d_elastic_create", "pf5d_stepper_create",
                 "pf5d_stepper_advance", "pf5d_adaptive_dt", "pf5d_oob_stats"]:
        assert name in syms


def test_library_exports_every_declared_symbol(lib):
    from phasefield5d_b200 import _lib
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    exported = set(re.findall(r"\sT\s(pf5d_\w+)", out))
    missing = [s for s in declared_symbols() if s not in exported]
    assert not missing, missing
    for s in declared_symbols():
        assert hasattr(lib, s)
    assert set(_lib.exported_symbols()) == set(declared_symbols())


def test_host_adaptive_dt_matches_reference(lib, kernels_golden):
    g = kernels_golden
    for c, want in zip(g["adt_cases"], g["adt_out"]):
        got = lib.pf5d_adaptive_dt(c[0], c[1], c[2], c[3], c[4], c[5], 2.0)
        assert got == want, (c, got, want)


def test_python_adaptive_dt_matches_reference(kernels_golden):
    from phasefield5d_b200.solver.system import apply_adaptive_time
    g = kernels_golden
    for c, want in zip(g["adt_cases"], g["adt_out"]):
        got = apply_adaptive_time(c[0], c[1], c[2], c[3], composition_change_lower_limit=c[4],
                                  composition_change_upper_limit=c[5])
        assert got == want


def test_gpu_entry_points_refuse_without_cuda():
    import torch
    if torch.cuda.is_available():
        pytest.skip("CUDA present")
    from phasefield5d_b200.solver import operators
    with pytest.raises(RuntimeError):
        operators.abs_max(np.ones(4))
