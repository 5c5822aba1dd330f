"""SolveConfig.from_simulation_config on SimulationConfig objects built by the
reference's own parse_args_to_config (tests/golden/sim_configs.json, written
by tests/golden/make_golden.py from phasefield5d/solver/config.py:146-184).

Each fixture case is rebuilt as an object with the dataclass's fields and
values (arrays as numpy arrays, as the parser leaves them) and handed to the
adapter unchanged; supported options map field by field, unsupported ones
raise ValueError.
"""
import json
import os
import types

import numpy as np
import pytest

from phasefield5d_b200 import workload as W

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "sim_configs.json")


def _cases():
    with open(GOLDEN) as f:
        d = json.load(f)
    out = []
    for c in d["cases"]:
        fields = dict(c["fields"])
        for k in c["arrays"]:
            fields[k] = np.asarray(fields[k], dtype=int if k == "direction" else float)
        out.append((c["argv"], types.SimpleNamespace(**fields), d["field_order"]))
    return out


CASES = _cases()


def test_fixture_has_every_simulation_config_field():
    for _, sim, order in CASES:
        assert sorted(vars(sim)) == sorted(order)


@pytest.mark.parametrize("idx", [0, 1, 2])
def test_supported_configs_map_field_by_field(idx):
    argv, sim, _ = CASES[idx]
    cfg = W.SolveConfig.from_simulation_config(sim)
    assert cfg.system_dim == sim.system_dim
    assert cfg.initial_composition == tuple(sim.initial_composition.reshape(-1))
    assert cfg.kappa_i == tuple(sim.kappa_i.reshape(-1))
    assert cfg.direction == tuple(int(v) for v in sim.direction)
    assert cfg.temperature == float(sim.temperature.rstrip("K"))
    for name in ("resolution", "fluctuation", "mw", "ppw", "kappa_value", "steps_per_ctld",
                 "total_timesteps", "lower_limit", "upper_limit", "safety",
                 "include_cubic_anisotropy", "time_linear_end_multiplier", "early_stage_frames",
                 "late_burst_duration_ctld", "late_burst_frames", "late_tail_frames",
                 "atomic_radius_tag"):
        assert getattr(cfg, name) == getattr(sim, name), name
    assert cfg.adaptive is True
    sched = cfg.save_schedule()
    assert sched["early_stage_frames"] == sim.early_stage_frames
    assert sched["late_tail_frames"] == sim.late_tail_frames


def test_overrides_apply_after_mapping():
    _, sim, _ = CASES[1]
    cfg = W.SolveConfig.from_simulation_config(sim, shape=(64, 48), omega_seed=4)
    assert cfg.shape == (64, 48) and cfg.omega_seed == 4
    with pytest.raises(ValueError):
        W.SolveConfig.from_simulation_config(sim, not_a_field=1)


@pytest.mark.parametrize("idx,what", [(3, "elements"), (4, "data_path"), (5, "load_path")])
def test_unsupported_options_raise(idx, what):
    _, sim, _ = CASES[idx]
    with pytest.raises(ValueError, match=what):
        W.SolveConfig.from_simulation_config(sim)


def test_bad_temperature_and_dimension_raise():
    _, sim, _ = CASES[0]
    bad = types.SimpleNamespace(**{**vars(sim), "temperature": "hot"})
    with pytest.raises(ValueError):
        W.SolveConfig.from_simulation_config(bad)
    bad = types.SimpleNamespace(**{**vars(sim), "system_dim": 4})
    with pytest.raises(ValueError):
        W.SolveConfig.from_simulation_config(bad)


def test_mapped_config_builds_a_problem():
    """The 2D case (the named 2D settings) builds through the same host setup
    as the named workload, to the same solve."""
    _, sim, _ = CASES[1]
    cfg = W.SolveConfig.from_simulation_config(sim, shape=(32, 32))
    named = W.config_2d_adaptive()
    named.shape = (32, 32)
    a, b = W.build_problem(cfg), W.build_problem(named)
    assert a.omega_seed == b.omega_seed
    assert a.ctld == b.ctld and a.dx == b.dx and a.t_cfl == b.t_cfl
    assert np.array_equal(a.X_init, b.X_init)
