"""Save-step host logic against the reference (tests/golden/save_io.json,
written by make_golden.py from phasefield5d/solver/io.py): the save schedule
decisions, the state-file format, the trace CSV; and the driver's look-ahead,
which must save at exactly the steps a per-step ``should_save`` loop saves."""
import json
import os

import numpy as np
import pytest

from phasefield5d_b200.solver import io as IO

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "save_io.json")


@pytest.fixture(scope="module")
def golden():
    with open(GOLDEN) as f:
        return json.load(f)


def _times(c):
    t, dt, out = 0.0, c["dt0"], []
    for _ in range(c["n"]):
        dt = min(dt * c["growth"], c["cap"])
        t = t + dt
        out.append(t)
    return out


def test_should_save_matches_reference(golden):
    for c in golden["schedule"]:
        data, snap = [], []
        for step, t in enumerate(_times(c)):
            d, s = IO.should_save(step, c["ctld"], t, c["n"], **c["kwargs"])
            if d:
                data.append(step)
            if s:
                snap.append(step)
        assert data == c["data_steps"]
        assert snap == c["snap_steps"]


def test_state_file_format(golden, tmp_path):
    X = np.arange(24, dtype=np.float64).reshape(3, 2, 4) / 100.0
    name = IO.save_current_state(str(tmp_path), 12, 1e-9, 3e-7, X)
    g = golden["npz"]
    assert os.path.basename(name) == g["name"]
    z = np.load(name)
    assert sorted(z.files) == g["keys"]
    for k in z.files:
        assert str(z[k].dtype) == g["dtypes"][k]
        assert list(z[k].shape) == g["shapes"][k]
    assert np.array_equal(z["current_composition"], X)


def test_trace_csv_matches_reference(golden, tmp_path):
    tr = IO.init_traces(4)
    IO.update_traces(tr, 5, 1e-7, 1e-9, 2e-9, np.arange(4) * 1e-3, 0.5, np.arange(4) * 0.1,
                     np.arange(4) + 1.0, np.arange(4) * 1e-18, np.arange(4) * 0.01,
                     np.arange(4) * 0.02 + 0.1, 0.3, np.arange(4) * 1e-6, -2e-20)
    IO.finalize_traces(str(tmp_path), tr)
    with open(tmp_path / "timeseries_info.csv") as f:
        assert f.read() == golden["trace_csv"]
    with open(tmp_path / "timeseries_info.json") as f:
        assert json.load(f) == golden["trace_info"]


class _Field:
    def __init__(self, a):
        self.a = a

    def cpu(self):
        return self

    def numpy(self):
        return self.a


class FakeStepper:
    """Device stepper stand-in: dt grows by `growth` per step up to `cap`
    (within the adaptive rule's bound), X is a constant small field."""

    def __init__(self, dt0, growth, cap):
        self.t, self.dt, self.k = 0.0, dt0, 0
        self.growth, self.cap = growth, cap
        self.X = np.full((4, 3, 4), 0.2)
        self.graph_steps = 0

    def _one(self):
        self.dt = min(self.dt * self.growth, self.cap)
        self.t = self.t + self.dt
        self.k += 1

    def state(self):
        return dict(time=self.t, dt=self.dt, step=self.k, halted=False)

    def advance(self, n):
        self.graph_steps += n
        for _ in range(n):
            self._one()

    def step_save(self):
        step = self.k
        self._one()
        z = np.zeros(4)
        return dict(net=z, max_change=z, total_flux=z, mass=z, comp_min=z, comp_max=z,
                    comp_var=z, comp_fe_min=0.0, f_grad=0.0, xdotmax=0.0, dt=self.dt,
                    time=self.t, step=step, halted=False)

    def field(self):
        return _Field(self.X)


def test_driver_lookahead_saves_exactly_like_per_step_loop(golden, tmp_path):
    from phasefield5d_b200.driver import run_simulation
    c = golden["schedule"][0]
    kw = c["kwargs"]
    st = FakeStepper(c["dt0"], c["growth"], c["cap"])
    traces, files = run_simulation(
        st, c["n"], str(tmp_path), ctld=c["ctld"], t_cfl=c["cap"],
        early_stage_frames=kw["early_frames"], late_burst_duration_ctld=kw["burst_duration_ctld"],
        late_burst_frames=kw["burst_frames"], late_tail_frames=kw["tail_dt_ctld"],
        save_every_n_steps_data=kw["save_every_n_steps_data"],
        save_every_n_steps_snap=kw["save_every_n_steps_snap"])
    assert traces["timestep"] == c["data_steps"]
    assert st.k == c["n"]
    assert st.graph_steps > c["n"] // 2            # most steps ran as graph blocks
    names = sorted(os.listdir(tmp_path / "data"))
    assert names[0] == "step_000000000.npz" or "_initial" in " ".join(names)
    assert len(files) == len(c["data_steps"]) + 2   # initial + saves + final
