"""Save-step host side: the data/snapshot schedule, the state files and the
scalar traces of a run (phasefield5d/solver/io.py).

* ``should_save`` keeps the reference's schedule and call convention
  (io.py:42-109): state lives on the function, is reset at step 0, and a
  step is saved when the time after it passes the next data / snapshot time
  of the current stage (early: the first CTLD; burst; tail), plus every
  50,000 / 100,000 steps and at the last step.
* ``save_current_state`` writes the same ``.npz`` keys and dtypes
  (io.py:208-216), so the reference's readers load these files.
* ``init_traces`` / ``update_traces`` / ``finalize_traces`` keep the trace
  columns and the CSV + JSON outputs (io.py:287-338).

Snapshot figures (matplotlib PNGs) are not produced here.
"""
from __future__ import annotations

import json
import os

import numpy as np


class SaveSchedule:
    """State of the time-based save schedule of one run."""

    def __init__(self, ctld, *, early_frames=100, burst_duration_ctld=100.0, burst_frames=800,
                 tail_dt_ctld=10.0, snapshot_factor=10):
        ctld = float(ctld)
        self.t_early_end = ctld
        self.t_burst_end = ctld * (1.0 + burst_duration_ctld)
        early = max(1, early_frames)
        self.dt_data_early = ctld / early
        self.dt_snap_early = ctld / max(1, early // snapshot_factor)
        burst = max(1, burst_frames)
        burst_time = self.t_burst_end - self.t_early_end
        self.dt_data_burst = burst_time / burst
        self.dt_snap_burst = burst_time / max(1, burst // snapshot_factor)
        self.dt_data_tail = max(1e-30, tail_dt_ctld * ctld)
        self.dt_snap_tail = self.dt_data_tail * snapshot_factor
        self.next_data = 0.0
        self.next_snap = 0.0

    def intervals(self, t):
        if t < self.t_early_end:
            return self.dt_data_early, self.dt_snap_early
        if t < self.t_burst_end:
            return self.dt_data_burst, self.dt_snap_burst
        return self.dt_data_tail, self.dt_snap_tail

    def decide(self, step, t, total_steps, every_data=50_000, every_snap=100_000):
        if step == total_steps - 1:
            return True, True
        dt_data, dt_snap = self.intervals(t)
        save_d = save_s = False
        if t >= self.next_data:
            while t >= self.next_data:
                self.next_data += dt_data
            save_d = True
        if t >= self.next_snap:
            while t >= self.next_snap:
                self.next_snap += dt_snap
            save_s = True
        if every_data and step % every_data == 0:
            save_d = True
        if every_snap and step % every_snap == 0:
            save_s = True
        return save_d, save_s

    def next_threshold(self):
        """Earliest time at which ``decide`` can return a save by time."""
        return min(self.next_data, self.next_snap)


def should_save(step: int, ctld: float, time: float, total_steps: int, *, early_frames: int = 100,
                burst_duration_ctld: float = 100.0, burst_frames: int = 800,
                tail_dt_ctld: float = 10.0, snapshot_factor: int = 10,
                save_every_n_steps_data: int | None = 50_000,
                save_every_n_steps_snap: int | None = 100_000):
    """(save_data, save_snapshot) for ``step`` whose update ends at ``time``
    (phasefield5d/solver/io.py:42-109)."""
    if getattr(should_save, "_state", None) is None or step == 0:
        should_save._state = SaveSchedule(ctld, early_frames=early_frames,
                                          burst_duration_ctld=burst_duration_ctld,
                                          burst_frames=burst_frames, tail_dt_ctld=tail_dt_ctld,
                                          snapshot_factor=snapshot_factor)
        return True, True
    return should_save._state.decide(step, time, total_steps, save_every_n_steps_data,
                                     save_every_n_steps_snap)


should_save._state = None


def save_current_state(path, timestep, time_increment, time, current_composition, postfix=""):
    """``{path}/data/step_{timestep:09d}{postfix}.npz`` with timestep (int64),
    time and dt (float64) and current_composition (float64, (*spatial, 4))."""
    os.makedirs(os.path.join(path, "data"), exist_ok=True)
    name = os.path.join(path, "data", f"step_{timestep:09d}{postfix}.npz")
    np.savez(name, timestep=np.int64(timestep), time=np.float64(time),
             dt=np.float64(time_increment),
             current_composition=np.asarray(current_composition, dtype=np.float64))
    return name


def init_traces(n_components):
    cols = ["timestep", "time", "dt", "t_cfl", "cfl_ratio", "net", "composition_change_max"]
    cols += [f"composition_change_max_s{j}" for j in range(n_components)]
    cols += ["mass", "total_flux"]
    cols += [f"comp_min_s{j}" for j in range(n_components)]
    cols += [f"comp_max_s{j}" for j in range(n_components)]
    cols += ["comp_fe_min"]
    cols += [f"comp_var_s{j}" for j in range(n_components)]
    cols += ["f_grad"]
    return {c: [] for c in cols}


def update_traces(traces, timestep, time, dt, t_cfl, net, composition_change_max,
                  composition_change_max_per_solute, mass, total_flux, comp_min, comp_max,
                  comp_fe_min, comp_var, f_grad):
    traces["timestep"].append(int(timestep))
    traces["time"].append(float(time))
    traces["dt"].append(float(dt))
    traces["t_cfl"].append(float(t_cfl))
    traces["cfl_ratio"].append(float(dt / t_cfl) if t_cfl > 0.0 else float("inf"))
    traces["net"].append(np.asarray(net).tolist())
    traces["composition_change_max"].append(float(composition_change_max))
    for j, v in enumerate(np.asarray(composition_change_max_per_solute).ravel()):
        traces[f"composition_change_max_s{j}"].append(float(v))
    traces["mass"].append(np.asarray(mass).tolist())
    traces["total_flux"].append(np.asarray(total_flux).tolist())
    for name, vals in (("comp_min", comp_min), ("comp_max", comp_max)):
        for j, v in enumerate(np.asarray(vals).ravel()):
            traces[f"{name}_s{j}"].append(float(v))
    traces["comp_fe_min"].append(float(comp_fe_min))
    for j, v in enumerate(np.asarray(comp_var).ravel()):
        traces[f"comp_var_s{j}"].append(float(v))
    traces["f_grad"].append(float(f_grad))


def finalize_traces(path, traces, filename="timeseries_info.csv"):
    """timeseries_info.csv (one row per save step) + timeseries_info.json."""
    import pandas as pd
    df = pd.DataFrame(traces)
    out = os.path.join(path, filename)
    df.to_csv(out, index=False)
    with open(os.path.join(path, "timeseries_info.json"), "w") as f:
        json.dump({"rows": len(df), "columns": list(df.columns)}, f, indent=2)
    return out
