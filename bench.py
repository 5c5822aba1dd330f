#!/usr/bin/env python
"""Benchmark the Cahn-Hilliard step loop on B200.

Default workload (N=1): plain FP64 2D 512x512, the 41^4 synthetic table at
873 K, elasticity on, adaptive dt -- one "step" is one explicit time step of
the whole field.  The composition field, rates and FFT buffers of this
workload fit in L2, so L2 is flushed (a 256 MiB write) between timed steps
and each step is timed alone with CUDA events on the launching stream.

Prints one JSON line.  Beside the headline it carries the rate stage's
roofline (algorithmic bytes over CUDA-event time, against the measured HBM
copy peak, with the DRAM traffic of the committed ncu capture), the per-stage
times, an end-to-end figure through the C ABI with the field copied in from
and out to pinned host memory every step, a CPU baseline (the oracle on a
bounded sample of the same workload), the SM clocks sampled during the timed
region, and -- at N=1, unless ``--forms none`` -- the other forms:
``forms.fp32c_same_workload`` (precision form + its accuracy report),
``forms.batch64`` (the 64-solve batched form against 64 plain FP64 steppers),
``forms.serving`` (p50/p99 time to solution at several Poisson rates),
``forms.3d256`` (the 3D 256^3 workload, 51^4 table, in both forms with their
rooflines and the 5,000-step accuracy report) and ``forms.1d1280`` (the 1D
1280 fixed-dt workload in both forms).

``--impl reference`` times the reference algorithm's CPU implementation (the
oracle restatement of the Numba kernels + scipy FFT, all host threads) on the
same workload and prints the same line with "impl": "reference".  Under
torchrun every rank runs an independent replica (the path has no cross-solve
exchange); value = all ranks' grid-point steps / the slowest rank's time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
if HERE not in sys.path:
    sys.path.insert(0, HERE)

# Algorithmic HBM bytes per grid-point step (FP64, elasticity on): state X
# read+written once (64), dX/dt written+read once (64), the misfit scalar's
# trip through the FFT pair (6 x 8).
STEP_BYTES_FP64 = 176
# Fused rate kernel per grid point: read X (32) and s' (8), write dX/dt (32).
RATE_BYTES_FP64 = 72
# FP32-compensated form: X - X0 as FP32 hi+lo read+written (64), dX/dt
# FP32 written+read (32), the FP32 misfit scalar through the FFT pair (24).
STEP_BYTES_FP32C = 120
# Its rate kernel: read D hi (16) and s' (4), write dX/dt (16).
RATE_BYTES_FP32C = 36
FALLBACK_HBM_GBS = 6650.0
L2_FLUSH_BYTES = 256 << 20

WORKLOADS = {
    "2d": ("plain FP64 2D 512x512, 41^4 table, elastic, adaptive dt", "config_2d_adaptive"),
    "1d": ("plain FP64 1D 1280, 41^4 table, elastic, fixed dt", "config_1d_fixed"),
    "3d": ("plain FP64 3D 256^3, 51^4 table, elastic, adaptive dt", "config_3d_precision"),
    "3d128": ("plain FP64 3D 128^3, 51^4 table, elastic, adaptive dt (profiling size)",
              "config_3d_precision", (128, 128, 128)),
}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="2d")
    ap.add_argument("--precision", choices=["fp64", "fp32c"], default="fp64",
                    help="plain FP64 (bit-faithful) or FP32-compensated form")
    ap.add_argument("--accuracy-steps", type=int, default=2000,
                    help="steps of the FP32c-vs-FP64 accuracy report")
    ap.add_argument("--cpu-steps", type=int, default=None,
                    help="steps in the CPU-baseline sample (default: --steps, the reference "
                         "arm's sample; at most as many as fit in about 20 s)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--forms", default="fp32c,batch,serve,3d,1d",
                    help="extra measurements at N=1 (comma list of fp32c, batch, serve, 3d, 1d; "
                         "'none')")
    ap.add_argument("--accuracy-steps-3d", type=int, default=5000,
                    help="steps of the 3D 256^3 FP32c-vs-FP64 accuracy report")
    ap.add_argument("--batch-steps", type=int, default=1000,
                    help="timed steps of the 64-solve batched form (and its FP64 comparison)")
    ap.add_argument("--serve-requests", type=int, default=12)
    ap.add_argument("--serve-rates", default="1,10,50", help="Poisson arrival rates, req/s")
    ap.add_argument("--serve-steps", type=int, default=2000)
    ap.add_argument("--ncu-range", action="store_true",
                    help="after warm-up, run one extra step (untimed) between cudaProfilerStart/"
                         "Stop, for ncu --profile-from-start off")
    return ap.parse_args()


def build_problem(name):
    from phasefield5d_b200 import workload as W
    cfg = getattr(W, WORKLOADS[name][1])()
    if len(WORKLOADS[name]) > 2:
        cfg.shape = WORKLOADS[name][2]
    return W.build_problem(cfg)


def measured_peak():
    path = os.path.join(HERE, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def committed_traffic(kernel, workload, precision):
    """DRAM bytes of one step's ``kernel`` stage (all its launches) on this
    workload from the committed ncu capture (profiles/traffic.json), or None
    when none was taken."""
    try:
        with open(os.path.join(HERE, "profiles", "traffic.json")) as f:
            ent = json.load(f)[kernel][f"{workload}_{precision}"]
        return float(ent["dram_bytes_per_launch"])
    except Exception:
        return None


class ClockSampler:
    """nvidia-smi clock/throttle samples every 200 ms.  ``start`` waits for a
    first sample and ``stop`` for one more after the timed region, so the
    samples bracket it even when the region is shorter than the period."""
    Q = ("timestamp,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    NAMES = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]

    def __init__(self, index):
        self.index = index
        self.path = tempfile.NamedTemporaryFile("w", suffix=".csv", delete=False).name
        self.p = None
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--id={index}", f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200",
                                       "-f", self.path], stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def _rows(self):
        try:
            with open(self.path) as f:
                return [[x.strip() for x in line.split(",")] for line in f
                        if line.count(",") >= 8]
        except OSError:
            return []

    def _wait_rows(self, n, timeout=3.0):
        t0 = time.time()
        while self.p is not None and len(self._rows()) < n and time.time() - t0 < timeout:
            time.sleep(0.05)

    def start(self):
        self._wait_rows(1)
        self.n0 = max(len(self._rows()) - 1, 0)
        return self

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self._wait_rows(len(self._rows()) + 1)
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except Exception:
            self.p.kill()
        rows = self._rows()[self.n0:]
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}

        def num(v):
            try:
                return float(v)
            except ValueError:
                return None
        sm = [v for v in (num(r[1]) for r in rows) if v is not None]
        mx = [v for v in (num(r[2]) for r in rows) if v is not None]
        reasons = sorted({self.NAMES[i] for r in rows for i in range(4) if r[5 + i] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(rows), "window": "samples bracketing the timed region"}


def reduce_max_over_ranks(values, world, device=None):
    """Max over ranks of each value (per-rank device times); identity at N=1.
    Every rank must call it, in the same order."""
    import torch
    t = torch.tensor(list(values), dtype=torch.float64, device=device)
    if world > 1:
        import torch.distributed as dist
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(v) for v in t.tolist()]


def replica_throughput(points, steps, world, max_ms):
    """Whole-job grid-point steps/s of `world` independent replicas of one
    solve, timed by the slowest rank."""
    return world * points * steps / (max_ms * 1e-3)


def cpu_threads():
    from oracle import oracle as O
    return O.num_threads()


def time_oracle(prob, steps, warmup, budget_s=None, min_s=0.0):
    """Reference algorithm on the host cores: (grid-point steps/s, seconds,
    steps timed).  The sample runs ``steps`` steps and keeps going until
    ``min_s`` seconds have passed; with ``budget_s`` it stops early once that
    much time has passed (at least one step is timed)."""
    from oracle.oracle import OracleStepper
    st = OracleStepper.from_problem(prob, fft_workers=-1)
    for _ in range(warmup):
        st.step()
    t0 = time.perf_counter()
    done = 0
    while done < steps or time.perf_counter() - t0 < min_s:
        st.step()
        done += 1
        if budget_s is not None and time.perf_counter() - t0 > budget_s:
            break
    dt = time.perf_counter() - t0
    return prob.n_points * done / dt, dt, done


def cpu_baseline(prob, args, workload_name, budget_s=20.0, min_s=10.0):
    """The oracle on the host cores, on a bounded sample of the workload:
    at least ``--cpu-steps`` (default ``--steps``) steps and 10 s of work,
    at most 20 s."""
    steps = args.cpu_steps if args.cpu_steps is not None else args.steps
    val, secs, done = time_oracle(prob, steps, 1, budget_s=budget_s, min_s=min_s)
    return {"value": val, "unit": "grid-point steps/s", "cores": cpu_threads(), "kind": "port",
            "sample": f"{done} steps ({secs:.1f} s) of the full {workload_name} after 1 warm-up "
                      f"(oracle C restatement + scipy FFT, all host threads)"}


def run_reference(args, rank):
    if rank != 0:
        return
    prob = build_problem(args.workload)
    value, secs, done = time_oracle(prob, args.steps, args.warmup)
    sample = f"{done} steps of the full {WORKLOADS[args.workload][0]} after {args.warmup} warm-up"
    line = {
        "impl": "reference", "metric": "grid-point steps/s", "value": value,
        "unit": "grid-point steps/s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * secs / done, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOADS[args.workload][0], "shape": list(prob.shape),
                   "parallelism": "cpu-threads"},
        "cpu_baseline": {"value": value, "unit": "grid-point steps/s", "cores": cpu_threads(),
                         "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": "grid-point steps/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def _events(torch):
    return torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)


def _stepper_timing(prob, precision, args, flush, torch):
    """Device-resident one-step timing with L2 flushed between steps, and the
    fused rate kernel launched alone: (ms per step, rate ms, variant)."""
    from phasefield5d_b200 import _lib
    from phasefield5d_b200.stepper import Stepper
    stream = torch.cuda.current_stream()
    st = Stepper.from_problem(prob, precision=precision)
    st.advance(1)
    for _ in range(args.warmup):
        flush.zero_()
        st.advance(1)
    ev = []
    for _ in range(args.steps):
        flush.zero_()
        a, b = _events(torch)
        a.record(stream)
        st.advance(1)
        b.record(stream)
        ev.append((a, b))
    torch.cuda.synchronize()
    step_ms = sum(a.elapsed_time(b) for a, b in ev) / len(ev)
    rate = []
    for _ in range(3):
        st.launch_stage(_lib.STAGE_RATE)
    for _ in range(max(args.steps, 10)):
        flush.zero_()
        a, b = _events(torch)
        a.record(stream)
        st.launch_stage(_lib.STAGE_RATE)
        b.record(stream)
        rate.append((a, b))
    torch.cuda.synchronize()
    rate_ms = sum(a.elapsed_time(b) for a, b in rate) / len(rate)
    variant, kernels = st.variant, st.rate_kernels
    st.close()
    return step_ms, rate_ms, variant, kernels


def form_workload(prob, workload, precision, args, flush, torch, accuracy_steps=0):
    """One workload in one form: device-resident steps timed alone with L2
    flushed between them, and the rate stage launched alone (its roofline:
    algorithmic bytes over CUDA-event time against the measured HBM peak,
    beside the DRAM traffic of the committed ncu capture).  With
    ``accuracy_steps`` (FP32c only) the accuracy report against the plain
    FP64 form over that many steps."""
    from phasefield5d_b200.precision import compare_forms
    peak, peak_kind = measured_peak()
    P = prob.n_points
    fp32c = precision == "fp32c"
    step_ms, rate_ms, variant, kernels = _stepper_timing(prob, precision, args, flush, torch)
    per_rate = RATE_BYTES_FP32C if fp32c else RATE_BYTES_FP64
    per_step = STEP_BYTES_FP32C if fp32c else STEP_BYTES_FP64
    if prob.lvec is None:
        per_rate -= 4 if fp32c else 8
        per_step -= 24 if fp32c else 48
    rate_bytes = per_rate * P
    value = P / (step_ms * 1e-3)
    achieved = rate_bytes / (rate_ms * 1e-3) / 1e9
    out = {"value": value, "unit": "grid-point steps/s", "ms_per_step": step_ms,
           "shape": list(prob.shape), "precision": precision,
           "l2": "flushed (256 MiB write) between timed steps", "rate_variant": variant,
           "roofline": {"bound": "hbm", "kernel": kernels, "ms_per_launch": rate_ms,
                        "achieved": achieved, "peak": peak, "peak_kind": peak_kind,
                        "unit": "GB/s", "frac": achieved / peak,
                        "algorithmic_bytes_per_launch": rate_bytes,
                        "traffic": committed_traffic("rate", workload, precision)},
           "step_roofline": {"bytes_per_grid_point_step": per_step,
                             "achieved_gbs": per_step * value / 1e9,
                             "frac": per_step * value / 1e9 / peak}}
    if fp32c and accuracy_steps > 0:
        out["accuracy_vs_fp64"] = compare_forms(prob, accuracy_steps)
    return out


def form_fp32c(prob, args, flush, torch):
    """FP32-compensated form on the headline workload, with its accuracy
    report against the plain FP64 form (max/RMS error, mass drift)."""
    return form_workload(prob, args.workload, "fp32c", args, flush, torch,
                         accuracy_steps=args.accuracy_steps)


def form_named(workload, args, flush, torch, accuracy_steps):
    """A named workload other than the headline's (``3d``: 3D 256^3 with the
    51^4 table, the one whose field exceeds L2; ``1d``: 1D 1280 at fixed dt)
    in the plain FP64 and FP32c forms, with FP32c's accuracy report."""
    prob = build_problem(workload)
    out = {"workload": WORKLOADS[workload][0]}
    for prec in ("fp64", "fp32c"):
        out[prec] = form_workload(prob, workload, prec, args, flush, torch,
                                  accuracy_steps=accuracy_steps if prec == "fp32c" else 0)
    out["speedup_fp32c_vs_fp64"] = out["fp32c"]["value"] / out["fp64"]["value"]
    return out


def profiled_step(torch, step, flush):
    """One untimed step between cudaProfilerStart / Stop (L2 flushed before),
    so that ncu --profile-from-start off captures exactly one step's kernels."""
    flush.zero_()
    torch.cuda.synchronize()
    torch.cuda.cudart().cudaProfilerStart()
    step()
    torch.cuda.synchronize()
    torch.cuda.cudart().cudaProfilerStop()


def form_batch(args, flush, torch):
    """The 64-solve batched FP32-compensated form (uneven 1D 2048-8192 and
    2D 128^2-384^2 grids, four temperature tables) against the plain FP64
    form on the same 64 solves, each on its own stream.  Both run the same
    steps; the accuracy report compares every solve's field afterwards."""
    from phasefield5d_b200 import workload as W
    from phasefield5d_b200.batch import BatchStepper
    from phasefield5d_b200.stepper import Stepper
    probs, _ = W.build_batched_problems(W.batched_configs(64))
    P = sum(p.n_points for p in probs)
    block = 50
    n_blocks = max(args.batch_steps // block, 1)
    n_warm = 3
    stream = torch.cuda.current_stream()

    b = BatchStepper(probs, stream=stream)
    for _ in range(n_warm):
        b.advance(block)
    ev = []
    for _ in range(n_blocks):
        flush.zero_()
        e0, e1 = _events(torch)
        e0.record(stream)
        b.advance(block)
        e1.record(stream)
        ev.append((e0, e1))
    torch.cuda.synchronize()
    batch_ms = sum(x.elapsed_time(y) for x, y in ev) / (n_blocks * block)

    streams = [torch.cuda.Stream() for _ in probs]
    singles = []
    for p, s in zip(probs, streams):
        with torch.cuda.stream(s):
            singles.append(Stepper.from_problem(p, precision="fp64", stream=s))
    torch.cuda.synchronize()

    def fp64_block():
        e0, e1 = _events(torch)
        e0.record(stream)
        for st, s in zip(singles, streams):
            s.wait_event(e0)
            st.advance(block)
            stream.wait_stream(s)
        e1.record(stream)
        return e0, e1

    for _ in range(n_warm):
        fp64_block()
    ev = []
    for _ in range(n_blocks):
        flush.zero_()
        ev.append(fp64_block())
    torch.cuda.synchronize()
    fp64_ms = sum(x.elapsed_time(y) for x, y in ev) / (n_blocks * block)

    errs, rms, drift = [], [], []
    states = b.states()
    for i, (p, st) in enumerate(zip(probs, singles)):
        if states[i]["halted"] or st.state()["halted"]:
            raise RuntimeError(f"batched solve {i} halted during the benchmark")
        xb = b.field(i).cpu().numpy().reshape(-1, 4)
        x64 = st.field().cpu().numpy().reshape(-1, 4)
        scale = np.max(np.abs(x64))
        errs.append(float(np.max(np.abs(xb - x64)) / scale))
        rms.append(float(np.sqrt(np.mean((xb - x64) ** 2)) / scale))
        drift.append(float(np.max(np.abs(xb.mean(axis=0) - p.X_init.reshape(-1, 4).mean(axis=0)))))
        st.close()
    variant, tuned = b.variant, b.tuned_ms
    if args.ncu_range:                  # after the comparison: it takes one more step
        profiled_step(torch, lambda: b.advance(1), flush)
    b.close()
    v_b = P / (batch_ms * 1e-3)
    v_64 = P / (fp64_ms * 1e-3)
    return {"solves": len(probs), "grid_points": P, "steps": (n_warm + n_blocks) * block,
            "timed_steps": n_blocks * block,
            "fp32c_batched": {"value": v_b, "unit": "grid-point steps/s", "ms_per_step": batch_ms,
                              "variant": variant, "tuned_rate_ms": tuned,
                              "bytes_per_grid_point_step": STEP_BYTES_FP32C,
                              "step_roofline_frac": STEP_BYTES_FP32C * v_b / 1e9 / measured_peak()[0]},
            "fp64_streams": {"value": v_64, "unit": "grid-point steps/s", "ms_per_step": fp64_ms,
                             "note": "64 plain FP64 steppers, one stream each, 50-step graphs"},
            "speedup_fp32c_batched_vs_fp64": v_b / v_64,
            "max_rel_err_vs_fp64": max(errs), "rms_rel_err_vs_fp64_max": max(rms),
            "mass_drift_max_fp32c": max(drift),
            "timing": "CUDA events around each 50-step graph launch, L2 flushed between blocks",
            "note": "the workload runs 10,000 steps per solve; a fixed number of steps is "
                    "timed (per-step cost does not depend on the step index)"}


def form_serve(args):
    """The serving form: Poisson streams of mixed 1D 4096 / 2D 256^2 / 3D
    64^3-192^3 requests at each rate, FP32-compensated continuous batching
    against one plain FP64 stepper per request."""
    import copy
    from phasefield5d_b200 import workload as W
    from phasefield5d_b200.serving import Request, Server, poisson_arrivals, serving_configs
    cfgs = serving_configs(args.serve_requests, seed=0, steps=args.serve_steps)
    probs, _ = W.build_batched_problems(cfgs)
    rates = [float(r) for r in args.serve_rates.split(",") if r]
    out = {"requests": len(probs), "steps_per_request": args.serve_steps,
           "mix": [list(p.shape) for p in probs], "rates": {}}
    warm_state = {}
    for prec in ("fp32c", "fp64"):           # untimed pass: tune each shape, load the tables
        warm = Server(precision=prec, reserve_bytes=1 << 30)
        for i, p in enumerate(probs):
            warm.submit(Request(rid=i, problem=p, n_steps=50, arrival=0.0))
        warm.run(timeout=600)
        be = warm.backend
        warm_state[prec] = (dict(be.variants), dict(be.tables), dict(be.table_mu))
    for rate in rates:
        arr = poisson_arrivals(rate, len(probs), seed=int(rate * 1000))
        row = {}
        for prec in ("fp32c", "fp64"):
            srv = Server(precision=prec, reserve_bytes=1 << 30)
            # a running server: tuned variants and tables already resident
            v, tabs, mus = warm_state[prec]
            srv.backend.variants, srv.backend.tables, srv.backend.table_mu = (
                dict(v), dict(tabs), dict(mus))
            for i, (p, a) in enumerate(zip(probs, arr)):
                srv.submit(Request(rid=i, problem=copy.copy(p), n_steps=args.serve_steps,
                                   arrival=float(a)))
            row[prec] = srv.run(timeout=900)
        out["rates"][f"{rate:g}"] = row
    out["timing"] = ("host clock: arrival to result on the host per request; "
                     "throughput = grid-point steps / (last result - first arrival)")
    return out


def run_ours(args, rank, world, local_rank):
    import torch
    import torch.distributed as dist
    from phasefield5d_b200 import _lib
    from phasefield5d_b200.stepper import Stepper

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    prob = build_problem(args.workload)
    P = prob.n_points
    stream = torch.cuda.current_stream()
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    fp32c = args.precision == "fp32c"
    # ---- device-resident steps, L2 flushed between timed steps -------------
    st = Stepper.from_problem(prob, precision=args.precision)
    st.advance(1)                       # captures the one-step graph
    for _ in range(args.warmup):
        flush.zero_()
        st.advance(1)
    if args.ncu_range:
        profiled_step(torch, lambda: st.advance(1), flush)
    barrier()
    clocks = ClockSampler(local_rank).start()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]
    for e0, e1 in ev:
        flush.zero_()
        e0.record(stream)
        st.advance(1)
        e1.record(stream)
    barrier()
    clock_info = clocks.stop()
    step_ms = [e0.elapsed_time(e1) for e0, e1 in ev]
    total_ms = sum(step_ms)
    launches_per_step = st.launches_per_step
    rate_kernels = st.rate_kernels
    state = st.state()
    if state["halted"]:
        raise RuntimeError(f"stepper halted during the benchmark: {state}")

    # ---- back-to-back steps from the 50-step graph (L2-warm, informational)
    st.advance(50)
    torch.cuda.synchronize()
    w0, w1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    w0.record(stream)
    st.advance(200)
    w1.record(stream)
    torch.cuda.synchronize()
    resident_ms = w0.elapsed_time(w1) / 200

    # ---- dominant kernel (fused rate) alone, L2 flushed, same stream -------
    probe = Stepper.from_problem(prob, precision=args.precision)
    stage_ms = {}
    stages = [("rate", _lib.STAGE_RATE), ("update", _lib.STAGE_UPDATE)]
    if prob.lvec is not None:
        stages += [("fft_fwd", _lib.STAGE_FFT_FWD), ("bmul", _lib.STAGE_BMUL),
                   ("fft_inv", _lib.STAGE_FFT_INV)]
    for name, sid in stages:
        for _ in range(3):
            probe.launch_stage(sid)
        times = []
        for _ in range(max(args.steps, 10)):
            flush.zero_()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            probe.launch_stage(sid)
            b.record(stream)
            times.append((a, b))
        torch.cuda.synchronize()
        stage_ms[name] = sum(x.elapsed_time(y) for x, y in times) / len(times)
    probe.close()

    # ---- end to end through the C ABI with host buffers --------------------
    host = torch.from_numpy(prob.X_init.copy()).pin_memory()
    e2e_st = Stepper.from_problem(prob, precision=args.precision)
    xdev = e2e_st.X

    def e2e_step():
        xdev.copy_(host, non_blocking=True)
        if fp32c:
            e2e_st.reset(e2e_st.state_dt, e2e_st.state_time)   # re-seed hi/lo from X
        e2e_st.advance(1)
        if fp32c:
            host.copy_(e2e_st.field(), non_blocking=True)
        else:
            host.copy_(xdev, non_blocking=True)

    e2e_st.state_dt, e2e_st.state_time = prob.dt0, 0.0
    for _ in range(max(args.warmup, 1)):
        e2e_step()
    torch.cuda.synchronize()
    e2e_ev = []
    for _ in range(args.steps):
        flush.zero_()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        e2e_step()
        b.record(stream)
        e2e_ev.append((a, b))
    torch.cuda.synchronize()
    e2e_ms = sum(a.elapsed_time(b) for a, b in e2e_ev)
    e2e_st.close()

    # ---- max over ranks -----------------------------------------------------
    total_ms, e2e_ms, resident_ms = reduce_max_over_ranks([total_ms, e2e_ms, resident_ms], world,
                                                          device=dev)
    if rank != 0:
        return

    value = replica_throughput(P, args.steps, world, total_ms)
    peak, peak_kind = measured_peak()
    per_rate = RATE_BYTES_FP32C if fp32c else RATE_BYTES_FP64
    per_step = STEP_BYTES_FP32C if fp32c else STEP_BYTES_FP64
    rate_bytes = per_rate * P if prob.lvec is not None else (per_rate - (4 if fp32c else 8)) * P
    achieved = rate_bytes / (stage_ms["rate"] * 1e-3) / 1e9
    cpu = None
    if not args.no_cpu_baseline and world == 1:        # the CPU baseline: N = 1 only
        cpu = cpu_baseline(prob, args, WORKLOADS[args.workload][0])
    line = {
        "metric": "grid-point steps/s", "value": value, "unit": "grid-point steps/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32+f64 (compensated)" if fp32c else "f64",
        "data": "synthetic",
        "config": {"workload": WORKLOADS[args.workload][0], "shape": list(prob.shape),
                   "precision": args.precision,
                   "table_nodes_per_axis": int(prob.grid.shape[0]), "omega_seed": prob.omega_seed,
                   "l2": "flushed (256 MiB write) between timed steps",
                   "parallelism": f"replicas x{world}" if world > 1 else "single solve"},
        "roofline": {"bound": "hbm", "kernel": rate_kernels,
                     "achieved": achieved, "peak": peak, "peak_kind": peak_kind, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": committed_traffic("rate", args.workload, args.precision),
                     "algorithmic_bytes_per_launch": rate_bytes,
                     "ms_per_launch": stage_ms["rate"]},
        "step_roofline": {"bytes_per_grid_point_step": per_step,
                          "achieved_gbs": per_step * value / world / 1e9,
                          "frac": per_step * value / world / 1e9 / peak},
        "stage_ms": stage_ms,
        "rate_variant": {"index": st.variant, "tuned_ms": st.tuned_ms,
                         "tuned_ms_is": "ms per step of the fastest whole-step graph (FP64 2D/3D)"
                                        if not fp32c and prob.dim > 1 else "ms per rate stage"},
        "resident_l2_warm": {"value": world * P / (resident_ms * 1e-3),
                             "ms_per_step": resident_ms,
                             "note": "200 back-to-back steps from 50-step graphs, no flush"},
        "cpu_baseline": cpu,
        "e2e": {"value": world * P * args.steps / (e2e_ms * 1e-3), "unit": "grid-point steps/s",
                "h2d_bytes_per_step": int(host.numel() * 8),
                "d2h_bytes_per_step": int(host.numel() * 8),
                "path": "pinned host X -> H2D -> pf5d_stepper_advance(1) -> D2H, per step"},
        "clocks": clock_info,
        "gpu_launches": args.steps * launches_per_step,
        "state_after": {"step": state["step"], "dt": state["dt"], "time": state["time"]},
    }
    if fp32c and args.accuracy_steps > 0:
        from phasefield5d_b200.precision import compare_forms
        line["accuracy_vs_fp64"] = compare_forms(prob, args.accuracy_steps)
    st.close()
    forms = [f for f in args.forms.split(",") if f and f != "none"]
    if world == 1 and forms:
        extra = {}
        if "fp32c" in forms and not fp32c:
            extra["fp32c_same_workload"] = form_fp32c(prob, args, flush, torch)
        if "batch" in forms:
            extra["batch64"] = form_batch(args, flush, torch)
        if "serve" in forms:
            extra["serving"] = form_serve(args)
        if "3d" in forms and args.workload != "3d":
            extra["3d256"] = form_named("3d", args, flush, torch, args.accuracy_steps_3d)
        if "1d" in forms and args.workload != "1d":
            extra["1d1280"] = form_named("1d", args, flush, torch, 10_000)
        line["forms"] = extra
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank)
        return
    import torch
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    try:
        run_ours(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.barrier()
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
