"""The main loop of examples/simulate.py:200-365 on the device stepper, with
the reference's save steps: initial state, a state file and a trace row at
every data save, an out-of-bounds state on a halt, the final state and the
trace files.

The save decision of a step needs the time after it, which the device
computes.  Reading it back every step would stall the step graphs, so the
loop looks ahead instead: dt can at most double per step and never exceeds
min(0.005 * ctld, t_cfl) (system.py:90-112), so the time after each of the
next k steps is bounded from above.  Steps whose bound stays below the next
save time of the schedule (and that are not a step-count save) cannot save
and run as graph blocks; the others run one at a time through
``Stepper.step_save`` and are decided by ``should_save`` with their actual
time, exactly as the reference decides them.
"""
from __future__ import annotations

from .solver.io import (finalize_traces, init_traces, save_current_state, should_save,
                        update_traces)


def _steps_below(time, dt, threshold, limit, *, adaptive, cap):
    """Largest k <= limit such that the time after each of the next k steps
    stays strictly below ``threshold``."""
    t, d, k = float(time), float(dt), 0
    while k < limit:
        d = min(2.0 * d, cap) if adaptive else d
        t = t + d
        if t * (1.0 + 1e-12) >= threshold:
            break
        k += 1
    return k


def run_simulation(stepper, total_steps, path, *, ctld, t_cfl, adaptive=True,
                   early_stage_frames=100, late_burst_duration_ctld=100, late_burst_frames=700,
                   late_tail_frames=300, save_every_n_steps_data=50_000,
                   save_every_n_steps_snap=100_000, max_block=50):
    """Run ``total_steps`` steps of ``stepper`` (either form) writing the
    reference's state files and traces under ``path``.  Returns the traces
    dict and the list of state files written."""
    kw = dict(early_frames=early_stage_frames, burst_duration_ctld=late_burst_duration_ctld,
              burst_frames=late_burst_frames, tail_dt_ctld=late_tail_frames, snapshot_factor=10,
              save_every_n_steps_data=save_every_n_steps_data,
              save_every_n_steps_snap=save_every_n_steps_snap)
    cap = min(0.005 * float(ctld), float(t_cfl))
    files = [save_current_state(path, 0, 0, 0.0, stepper.field().cpu().numpy(),
                                postfix="_initial")]
    traces = init_traces(4)
    should_save._state = None
    st = stepper.state()
    timestep = st["step"]
    last = max(total_steps - 1, 0)
    while timestep < total_steps:
        if st["halted"]:
            files.append(save_current_state(path, timestep, st["dt"], st["time"],
                                            stepper.field().cpu().numpy(),
                                            postfix="_out_of_bound"))
            last = timestep
            break
        k = 0
        if timestep > 0 and should_save._state is not None:
            limit = total_steps - 1 - timestep
            for every in (save_every_n_steps_data, save_every_n_steps_snap):
                if every:
                    limit = min(limit, (-timestep) % every)
            limit = min(limit, max_block)
            k = _steps_below(st["time"], st["dt"], should_save._state.next_threshold(), limit,
                             adaptive=adaptive, cap=cap)
        if k > 0:
            stepper.advance(k)
            st = stepper.state()
            timestep = st["step"]
            continue
        d = stepper.step_save()
        if d["halted"]:
            st = stepper.state()
            timestep = st["step"]
            continue
        save_data, _snap = should_save(timestep, ctld, d["time"], total_steps, **kw)
        if save_data:
            files.append(save_current_state(path, timestep, d["dt"], d["time"],
                                            stepper.field().cpu().numpy()))
            update_traces(traces, timestep, d["time"], d["dt"], t_cfl, d["net"], d["xdotmax"],
                          d["max_change"], d["mass"], d["total_flux"], d["comp_min"],
                          d["comp_max"], d["comp_fe_min"], d["comp_var"], d["f_grad"])
        st = stepper.state()
        timestep = st["step"]
    # final save (after a halt too, as the reference's loop falls through)
    files.append(save_current_state(path, last, st["dt"], st["time"],
                                    stepper.field().cpu().numpy()))
    finalize_traces(path, traces)
    return traces, files
