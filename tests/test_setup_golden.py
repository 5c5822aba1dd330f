"""Host setup (phasefield5d_b200.workload / solver.system / elastic_setup) must
produce the reference's setup scalars for the named workloads: CTLD, dominant
wavenumber, dx, CFL bound, nominal Δt, rank-1 elastic factor, B(k) and the
seeded initial field.  CPU only."""
import hashlib
import json
import os

import numpy as np
import pytest

from phasefield5d_b200 import workload as W


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


@pytest.fixture(scope="module")
def setup_golden():
    with open(os.path.join(os.path.dirname(__file__), "golden", "setup.json")) as f:
        return json.load(f)


@pytest.mark.parametrize("name,mk", [("1d_fixed", W.config_1d_fixed),
                                     ("2d_adaptive", W.config_2d_adaptive),
                                     ("3d_precision", W.config_3d_precision)])
def test_setup_matches_reference(setup_golden, name, mk):
    ref = setup_golden[name]
    prob = W.build_problem(mk())
    assert prob.omega_seed == ref["omega_seed"]
    if sha(prob.table.data) != ref["table_sha"]:
        pytest.skip("synthetic table differs on this host (platform exp rounding)")
    assert sha(prob.grid) == ref["grid_sha"]
    assert prob.ctld == pytest.approx(ref["ctld"], rel=1e-13)
    assert prob.wavenumber_max == pytest.approx(ref["wavenumber_max"], rel=1e-13)
    assert prob.dx == ref["dx"]
    assert list(prob.shape) == ref["shape"]
    assert prob.t_cfl == ref["t_cfl"]
    assert prob.hessian_max == ref["hessian_max"]
    assert prob.mobility_max == ref["mobility_max"]
    assert np.array_equal(prob.lvec, np.array(ref["lvec"]))
    assert sha(prob.bk) == ref["bk_sha"]
    assert sha(prob.X_init) == ref["X_init_sha"]
    from phasefield5d_b200.solver.system import get_time_increment
    assert get_time_increment(prob.ctld, prob.cfg.steps_per_ctld) == ref["dt_nominal"]


def test_unstable_seed_rejection_is_recorded():
    prob = W.build_problem(W.config_1d_fixed())
    assert prob.rejected_seeds == list(range(0, prob.omega_seed))
    assert prob.ctld > 0


def test_stable_composition_raises():
    from phasefield5d_b200.solver.system import compute_initial_kinetics
    from phasefield5d_b200.solver.table import host_table_eval
    cfg = W.config_1d_fixed()
    table = W.make_table(cfg.resolution, cfg.temperature, 0)
    prob_grid = __import__("phasefield5d_b200.solver.table", fromlist=["x"]).build_4d_grid(
        table.data, cfg.resolution)[1]
    with pytest.raises(ValueError):
        compute_initial_kinetics(cfg.initial_composition, cfg.resolution, cfg.kappa_value,
                                 np.ones((1, 4)),
                                 lambda p: host_table_eval(p, prob_grid, cfg.resolution),
                                 n_k=500)
