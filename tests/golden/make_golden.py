"""Generate golden vectors by running the phasefield5d reference itself.

Run in a container where the reference source tree is available:

    python tests/golden/make_golden.py --ref /path/to/phasefield5d

It imports the reference read-only (with the import-only matplotlib stand-in
in ``_mplstub``), feeds its hot-path functions seeded inputs, and writes:

* ``table_small.npz``  -- the 0.05-spacing synthetic table the small cases use;
* ``kernels.npz``      -- per-kernel inputs and outputs (interpolation with the
                          nearest-row fallback, Laplacian, fused divergence,
                          gradients/fluxes, elastic update, abs_max, clamp,
                          adaptive Δt, out_of_bounds, initial condition);
* ``trajectories.npz`` -- small 1D/2D/3D step-loop runs in the order of
                          examples/simulate.py:242-320, per-step Δt and
                          max|dX/dt| recorded;
* ``setup.json``       -- the reference's setup scalars (CTLD, dx, CFL bound,
                          rank-1 factor, B(k) samples) for the named workloads;
* ``fullres.json``     -- SHA-256 digests of reference outputs at the full
                          41^4-table resolution (1D 1280 and 2D 512² steps),
                          guarded by a digest of the regenerated table;
* ``sim_configs.json`` -- SimulationConfig objects parsed by the reference's
                          own parse_args_to_config from seeded command lines.

Tables come from ``phasefield5d_b200.workload.make_table`` (the synthetic
regular-solution table), so the same inputs can be rebuilt by the tests.
"""
from __future__ import annotations

import argparse
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)

from phasefield5d_b200 import workload as W  # noqa: E402

SMALL_RES = 0.05
SMALL_X0 = (0.1, 0.2, 0.2, 0.25)
SMALL_T = 873.0


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def import_reference(ref):
    sys.path.insert(0, os.path.join(HERE, "_mplstub"))
    sys.path.insert(0, ref)
    import phasefield5d.solver.interpolation as I
    import phasefield5d.solver.operators as O
    import phasefield5d.solver.fluxes as F
    import phasefield5d.solver.elastic as E
    import phasefield5d.solver.system as S
    import phasefield5d.elasticity.anisotropy as A
    import phasefield5d.elasticity.energies as EN
    return dict(I=I, O=O, F=F, E=E, S=S, A=A, EN=EN)


class _Cfg:
    include_cubic_anisotropy = True

    def __init__(self, x0):
        self.initial_composition = np.asarray(x0, dtype=float)


def ref_setup(R, cfg, table):
    """Reference setup chain of examples/simulate.py:68-192 on a synthetic table."""
    I, S, E, A, EN = R["I"], R["S"], R["E"], R["A"], R["EN"]
    df = table.dataframe()
    _, grid = I.build_4d_grid(df, cfg.resolution)
    tree, vals = I.build_calphad_kdtree(df)
    X0 = np.asarray(cfg.initial_composition, dtype=float)
    ref = I.interpolator_nb(X0[None, :], grid, resolution=cfg.resolution, tree=tree,
                            calphad_values=vals)[0]
    hmax = float(np.abs(ref[:4]).max())
    mmax = float(ref[4:].max())
    eta = np.random.default_rng(cfg.misfit_seed).uniform(-0.02, 0.02, size=4)
    vm = EN.calculate_molar_volume(X0, W.MOLAR_VOLUMES_FEMNNICOCU)
    lam = np.outer(eta, eta)
    lam *= vm
    b_n, _ = A.calculate_khachaturyan_elastic_anisotropy(np.asarray(cfg.direction), cfg.c11,
                                                         cfg.c12, cfg.c44)
    el_mat = np.outer(eta, eta) * b_n * 1e9 * vm
    ctld, kmax = S.compute_initial_kinetics(
        initial_composition=X0, resolution=cfg.resolution, kappa_value=cfg.kappa_value,
        kappa_i=np.asarray(cfg.kappa_i, dtype=float).reshape(1, 4), data_grid=grid, tree=tree,
        calphad_values=vals, elastic_matrix=el_mat, n_k=cfg.n_k)
    dt_nom = S.get_time_increment(ctld, cfg.steps_per_ctld)
    _, dx, _, ncells = S.get_system_dimensions(kmax, ppw=cfg.ppw, mw=cfg.mw, dim=cfg.system_dim)
    shape = tuple(cfg.shape) if cfg.shape is not None else ncells
    t_cfl = S.cahn_hilliard_cfl_dt(dx, mmax, hmax, cfg.kappa_value, cfg.safety)
    if cfg.system_dim == 1:
        kg, kn = S.build_fourier_grid_1d_along_direction(shape[0], dx, cfg.direction)
    elif cfg.system_dim == 2:
        kg, kn = S.build_fourier_grid_2d_in_plane(shape[0], shape[1], dx, cfg.direction)
    else:
        kg, kn = S.build_fourier_grid_3d(shape[0], shape[1], shape[2], dx)
    bk = E.build_khachaturyan_kernel(kg, kn, cfg.c11, cfg.c12, cfg.c44)
    eigvals, eigvecs = np.linalg.eigh(lam)
    lvec = eigvecs[:, -1] * np.sqrt(eigvals[-1])
    np.random.seed(cfg.ic_seed)
    X = S.apply_fluctuations(X0, shape, cfg.fluctuation).astype(np.float64)
    return dict(grid=grid, tree=tree, vals=vals, X0=X0, hmax=hmax, mmax=mmax, eta=eta, vm=vm,
                lam=lam, ctld=ctld, kmax=kmax, dt_nom=dt_nom, dx=dx, shape=shape, t_cfl=t_cfl,
                bk=bk, lvec=lvec, X=X)


def ref_run(R, cfg, st, n_steps):
    """Reference loop body (examples/simulate.py:230-320), saves off."""
    I, O, F, E, S = R["I"], R["O"], R["F"], R["E"], R["S"]
    X = st["X"].copy()
    sp = X.shape[:-1]
    dim = len(sp)
    interp = np.empty((*sp, 9))
    lap = np.empty_like(X)
    dX = np.empty_like(X)
    mask = np.empty(int(np.prod(sp)), dtype=np.bool_)
    upd = E.make_elastic_updater(_Cfg(cfg.initial_composition), st["lam"], st["bk"], X.shape,
                                 np.float64)
    div = F.get_divergence_from_mu_function(dim)
    kappa = np.asarray(cfg.kappa_i, dtype=float).reshape(1, 4) * cfg.kappa_value
    inv_dx = 1.0 / st["dx"]
    if cfg.adaptive:
        dt = st["dt_nom"]
    else:
        dt = min(st["dt_nom"], 0.005 * st["ctld"], st["t_cfl"])
    time = 0.0
    dts, xds = [], []
    for step in range(n_steps):
        if step % 100 == 0 and S.out_of_bounds(X):
            break
        I.interpolator_nb(X, st["grid"], resolution=cfg.resolution, tree=st["tree"],
                          calphad_values=st["vals"], out=interp, mask_buffer=mask)
        mu = interp[..., :4]
        M = interp[..., 4:]
        O.calculate_laplacian(X, st["dx"], lap)
        lap *= kappa
        mu -= lap
        upd(mu, X)
        div(X, M, mu, inv_dx, dX)
        xd = float(O.abs_max(dX))
        if cfg.adaptive:
            dt = S.apply_adaptive_time(dt, xd, st["ctld"], st["t_cfl"],
                                       composition_change_lower_limit=cfg.lower_limit,
                                       composition_change_upper_limit=cfg.upper_limit)
        time += dt
        dX *= dt
        X += dX
        O.clamp_simplex(X)
        dts.append(dt)
        xds.append(xd)
    return X, np.array(dts), np.array(xds), time


def small_cfg(dim, shape, adaptive=True, ic_seed=2):
    return W.SolveConfig(system_dim=dim, initial_composition=SMALL_X0, resolution=SMALL_RES,
                         temperature=SMALL_T, kappa_value=5e-16, mw=4, ppw=16, shape=shape,
                         adaptive=adaptive, ic_seed=ic_seed, n_k=2000)


def gen_kernels(R, table, out_path):
    I, O, F, E, S = R["I"], R["O"], R["F"], R["E"], R["S"]
    rng = np.random.default_rng(20260101)
    df = table.dataframe()
    _, grid = I.build_4d_grid(df, SMALL_RES)
    tree, vals = I.build_calphad_kdtree(df)
    g = {"resolution": SMALL_RES, "grid_sha": sha(grid)}

    # --- interpolation: a smooth field near X0, random simplex points (some
    # in the nearest-row region), negative coordinates and exact nodes.
    field = np.asarray(SMALL_X0) + rng.uniform(-0.03, 0.03, size=(12, 12, 4))
    rnd = rng.dirichlet(np.ones(5), size=300)[:, 1:]
    edge = np.array([[-0.01, 0.1, 0.1, 0.1], [0.0, 0.0, 0.0, 0.0], [0.1, 0.2, 0.1, 0.1],
                     [0.3, 0.0, 0.0, 0.3], [1.0, 0.0, 0.0, 0.0], [0.25, 0.25, 0.05, 0.05],
                     [0.15, 0.15, 0.15, 0.15 - 1e-12], [0.2, 0.2, 0.1, 0.1000000001]])
    pts = np.concatenate([field.reshape(-1, 4), rnd, edge], axis=0)
    out = np.empty((pts.shape[0], 9))
    mask = np.empty(pts.shape[0], dtype=np.bool_)
    I.interpolator_nb(pts, grid, resolution=SMALL_RES, tree=tree, calphad_values=vals, out=out,
                      mask_buffer=mask)
    g.update(interp_points=pts, interp_out=out, interp_mask=mask)

    # --- Laplacian, divergence, gradients/fluxes on non-cubic shapes.
    shapes = {1: (33,), 2: (9, 7), 3: (5, 6, 7)}
    dx = 1.3e-9
    for d, sh in shapes.items():
        X = np.asarray(SMALL_X0) + rng.uniform(-0.02, 0.02, size=(*sh, 4))
        lap = O.calculate_laplacian(X, dx)
        buf = np.empty((*sh, 9))
        buf[..., :4] = rng.uniform(-2e3, 2e3, size=(*sh, 4)) + 1e4
        buf[..., 4:] = np.exp(rng.normal(-30.0, 0.5, size=(*sh, 5)))
        mu, M = buf[..., :4], buf[..., 4:]
        dX = np.empty_like(X)
        F.get_divergence_from_mu_function(d)(X, M, mu, 1.0 / dx, dX)
        gp, gm = O.calculate_gradients_pm(mu, dx)
        fp = np.empty_like(gp)
        fm = np.empty_like(gm)
        F.get_flux_function(d)(X, M, gp, gm, fp, fm)
        g.update({f"lap{d}_X": X, f"lap{d}_out": lap, f"div{d}_buf": buf, f"div{d}_out": dX,
                  f"grad{d}_p": gp, f"grad{d}_m": gm, f"flux{d}_p": fp, f"flux{d}_m": fm})
    g["dx"] = dx

    # --- elastic update (rank-1 scipy path) per dimension.
    eta = rng.uniform(-0.02, 0.02, size=4)
    lam = np.outer(eta, eta) * 7e-6
    for d, sh in {1: (40,), 2: (12, 10), 3: (6, 8, 5)}.items():
        if d == 1:
            kg, kn = S.build_fourier_grid_1d_along_direction(sh[0], dx, [1, 0, 0])
        elif d == 2:
            kg, kn = S.build_fourier_grid_2d_in_plane(sh[0], sh[1], dx, [1, 0, 0])
        else:
            kg, kn = S.build_fourier_grid_3d(*sh, dx)
        bk = E.build_khachaturyan_kernel(kg, kn, 240.0, 150.0, 120.0)
        X = np.asarray(SMALL_X0) + rng.uniform(-0.02, 0.02, size=(*sh, 4))
        mu = rng.uniform(-1e3, 1e3, size=(*sh, 4))
        mu_in = mu.copy()
        E.make_elastic_updater(_Cfg(SMALL_X0), lam, bk, X.shape, np.float64)(mu, X)
        ev, evec = np.linalg.eigh(lam)
        g.update({f"el{d}_X": X, f"el{d}_bk": bk, f"el{d}_mu_in": mu_in, f"el{d}_mu_out": mu,
                  f"el{d}_lvec": evec[:, -1] * np.sqrt(ev[-1])})
    g["el_X0"] = np.asarray(SMALL_X0)

    # --- reductions, clamp, adaptive Δt, out_of_bounds, initial condition.
    a = rng.normal(size=(17, 13, 4))
    a[3, 4, 1] = np.nan
    a[5, 5, 2] = -7.5
    g.update(absmax_in=a, absmax_out=O.abs_max(a))
    Xc = rng.uniform(0.0, 0.4, size=(50, 4))
    Xc_out = Xc.copy()
    O.clamp_simplex(Xc_out)
    g.update(clamp_in=Xc, clamp_out=Xc_out)
    cases = [(1e-5, 1e3, 1.0, 1e-2, 1e-5, 1e-3), (3e-9, 0.0, 3.8e-6, 2.6e-12, 1e-5, 1e-3),
             (3e-9, 12.5, 3.8e-6, 2.6e-12, 1e-5, 1e-3), (2e-12, 1e4, 1e-6, 1e-9, 1e-5, 1e-3),
             (2e-12, 1e7, 1e-6, 1e-9, 1e-5, 1e-3), (1e-10, 1e2, 1e-6, 1e-9, 1e-3, 1e-5),
             (5e-11, np.inf, 1e-6, 1e-9, 1e-5, 1e-3), (5e-11, 3.3e5, 1e-9, 1.0, 1e-5, 1e-3)]
    res = [S.apply_adaptive_time(c[0], c[1], c[2], c[3], composition_change_lower_limit=c[4],
                                 composition_change_upper_limit=c[5]) for c in cases]
    g.update(adt_cases=np.array(cases), adt_out=np.array(res))
    oob_in = []
    base = np.full((16, 4), 0.1)
    for mod in [None, (5, 2, np.nan), (1, 1, -2e-3), (2, 0, 1.0 + 2e-3), (3, 3, -5e-6),
                (4, 0, 0.8), (6, 1, np.inf)]:
        x = base.copy()
        if mod is not None:
            x[mod[0], mod[1]] = mod[2]
        oob_in.append(x)
    g.update(oob_in=np.array(oob_in), oob_out=np.array([bool(S.out_of_bounds(x)) for x in oob_in]))
    np.random.seed(7)
    g["ic_out"] = S.apply_fluctuations(np.asarray(SMALL_X0), (6, 5), 1e-3)
    np.savez_compressed(out_path, **g)


def gen_trajectories(R, table, out_path):
    runs = {"1d_fixed": (small_cfg(1, (48,), adaptive=False), 300),
            "1d_adapt": (small_cfg(1, (40,), adaptive=True), 300),
            "2d_adapt": (small_cfg(2, (12, 10)), 100),
            "3d_adapt": (small_cfg(3, (6, 5, 4)), 30)}
    g = {"resolution": SMALL_RES}
    for name, (cfg, n) in runs.items():
        st = ref_setup(R, cfg, table)
        X, dts, xds, time = ref_run(R, cfg, st, n)
        g.update({f"{name}_X_init": st["X"], f"{name}_X_final": X, f"{name}_dts": dts,
                  f"{name}_xdotmax": xds, f"{name}_time": time, f"{name}_bk": st["bk"],
                  f"{name}_lvec": st["lvec"], f"{name}_X0": st["X0"],
                  f"{name}_scalars": np.array([st["dx"], st["ctld"], st["t_cfl"], st["dt_nom"],
                                               cfg.kappa_value, float(cfg.adaptive), n,
                                               cfg.lower_limit, cfg.upper_limit])})
    np.savez_compressed(out_path, **g)


def gen_setup(R):
    out = {}
    for name, mk in [("1d_fixed", W.config_1d_fixed), ("2d_adaptive", W.config_2d_adaptive),
                     ("3d_precision", W.config_3d_precision)]:
        cfg = mk()
        prob = W.build_problem(cfg)
        st = ref_setup(R, cfg, prob.table)
        out[name] = dict(
            omega_seed=prob.table.seed, table_sha=sha(prob.table.data), ctld=st["ctld"],
            wavenumber_max=st["kmax"], dx=st["dx"], shape=list(st["shape"]), t_cfl=st["t_cfl"],
            dt_nominal=st["dt_nom"], hessian_max=st["hmax"], mobility_max=st["mmax"],
            lvec=st["lvec"].tolist(), bk_sum=float(np.sum(st["bk"])),
            bk_first=np.asarray(st["bk"]).reshape(-1)[:8].tolist(), bk_sha=sha(st["bk"]),
            X_init_sha=sha(st["X"]), grid_sha=sha(st["grid"]))
    return out


def gen_fullres(R):
    out = {}
    for name, mk, shape, n in [("1d_fixed_1280", W.config_1d_fixed, None, 200),
                               ("2d_adaptive_512", W.config_2d_adaptive, None, 20)]:
        cfg = mk()
        prob = W.build_problem(cfg)
        st = ref_setup(R, cfg, prob.table)
        interp = R["I"].interpolator_nb(st["X"], st["grid"], resolution=cfg.resolution,
                                        tree=st["tree"], calphad_values=st["vals"])
        X, dts, xds, time = ref_run(R, cfg, st, n)
        out[name] = dict(table_sha=sha(prob.table.data), X_init_sha=sha(st["X"]), steps=n,
                         interp_sha=sha(interp), X_final_sha=sha(X), dts_sha=sha(dts),
                         time=time, xdotmax_last=float(xds[-1]),
                         X_final_sum=float(np.sum(X)))
    return out


def schedule_times(n, ctld, dt0, growth, cap):
    """A time series with geometric dt growth up to a cap (as the adaptive
    rule produces), used to exercise every stage of the save schedule."""
    t, dt, out = 0.0, dt0, []
    for _ in range(n):
        dt = min(dt * growth, cap)
        t = t + dt
        out.append(t)
    return out


SCHEDULE_CASES = [
    # (n steps, ctld, dt0, growth, cap, should_save kwargs)
    (3000, 1e-6, 1e-12, 1.01, 0.005e-6, dict(early_frames=7, burst_duration_ctld=3.0,
                                              burst_frames=11, tail_dt_ctld=0.2,
                                              snapshot_factor=10, save_every_n_steps_data=700,
                                              save_every_n_steps_snap=1500)),
    (30000, 2e-7, 1e-14, 1.05, 1e-9, dict(early_frames=100, burst_duration_ctld=100,
                                          burst_frames=700, tail_dt_ctld=300,
                                          snapshot_factor=10)),
]


def gen_save(ref, out_path):
    """Save-step host logic of the reference (phasefield5d/solver/io.py):
    should_save decisions over seeded time series, the state-file keys and
    dtypes, and the trace columns."""
    import tempfile
    import phasefield5d.solver.io as IO
    cases = []
    for n, ctld, dt0, growth, cap, kw in SCHEDULE_CASES:
        times = schedule_times(n, ctld, dt0, growth, cap)
        data, snap = [], []
        for step, t in enumerate(times):
            d, sn = IO.should_save(step, ctld, t, n, **kw)
            if d:
                data.append(step)
            if sn:
                snap.append(step)
        cases.append(dict(n=n, ctld=ctld, dt0=dt0, growth=growth, cap=cap, kwargs=kw,
                          data_steps=data, snap_steps=snap))
    with tempfile.TemporaryDirectory() as tmp:
        os.makedirs(os.path.join(tmp, "data"))
        X = np.arange(24, dtype=np.float64).reshape(3, 2, 4) / 100.0
        IO.save_current_state(tmp, 12, 1e-9, 3e-7, X)
        name = os.listdir(os.path.join(tmp, "data"))[0]
        z = np.load(os.path.join(tmp, "data", name))
        npz = dict(name=name, keys=sorted(z.files),
                   dtypes={k: str(z[k].dtype) for k in z.files},
                   shapes={k: list(z[k].shape) for k in z.files})
        tr = IO.init_traces(4)
        IO.update_traces(tr, 5, 1e-7, 1e-9, 2e-9, np.arange(4) * 1e-3, 0.5, np.arange(4) * 0.1,
                         np.arange(4) + 1.0, np.arange(4) * 1e-18, np.arange(4) * 0.01,
                         np.arange(4) * 0.02 + 0.1, 0.3, np.arange(4) * 1e-6, -2e-20)
        IO.finalize_traces(tmp, tr)
        with open(os.path.join(tmp, "timeseries_info.csv")) as f:
            csv_text = f.read()
        with open(os.path.join(tmp, "timeseries_info.json")) as f:
            info = json.load(f)
    with open(out_path, "w") as f:
        json.dump(dict(schedule=cases, npz=npz, trace_csv=csv_text, trace_info=info), f, indent=1)


# Command lines of examples/simulate.py whose parsed SimulationConfig the
# adapter test replays: the defaults, the named workloads' settings, and
# options the adapter must reject.
CONFIG_ARGVS = [
    [],
    ["--system_dim", "2", "--resolution", "0.025", "--initial_composition", "0.1,0.2,0.3,0.2",
     "--mw", "32", "--ppw", "16", "--kappa_value", "7.6e-15", "--total_timesteps", "20000"],
    ["--system_dim", "3", "--resolution", "0.02", "--mw", "16", "--kappa_i", "1,0.5,2,1",
     "--direction", "1,1,0", "--temperature", "973K", "--no_include_cubic_anisotropy",
     "--lower_limit", "2e-5", "--upper_limit", "5e-4", "--safety", "0.05",
     "--early_stage_frames", "50", "--late_burst_duration_ctld", "40",
     "--late_burst_frames", "300", "--late_tail_frames", "200", "--threads", "8",
     "--fft_workers", "-1", "--time_linear_end_multiplier", "50"],
    ["--elements", "Fe,Cr,Ni,Co,Mn"],
    ["--data_path", "data/FeMnNiCoCu_fcc"],
    ["--load_path", "run/data/state_000100.npz"],
]


def gen_configs(ref, out_path):
    """SimulationConfig objects built by the reference's own
    parse_args_to_config (phasefield5d/solver/config.py:146-184), stored as
    field dicts (arrays as nested lists)."""
    import dataclasses
    import importlib.util
    spec = importlib.util.spec_from_file_location(
        "pf5d_ref_config", os.path.join(ref, "phasefield5d", "solver", "config.py"))
    C = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(C)
    cases = []
    for argv in CONFIG_ARGVS:
        cfg = C.parse_args_to_config(argv)
        fields = {}
        for f in dataclasses.fields(cfg):
            v = getattr(cfg, f.name)
            fields[f.name] = v.tolist() if isinstance(v, np.ndarray) else v
        arrays = [f.name for f in dataclasses.fields(cfg)
                  if isinstance(getattr(cfg, f.name), np.ndarray)]
        cases.append(dict(argv=argv, fields=fields, arrays=arrays))
    with open(out_path, "w") as f:
        json.dump(dict(field_order=[f.name for f in dataclasses.fields(C.SimulationConfig)],
                       cases=cases), f, indent=1)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("PHASEFIELD5D_REF"),
                    help="path of the phasefield5d source tree (default: $PHASEFIELD5D_REF)")
    ap.add_argument("--only-save", action="store_true",
                    help="regenerate only the save-step host logic fixture")
    ap.add_argument("--only-configs", action="store_true",
                    help="regenerate only the parsed SimulationConfig fixture")
    args = ap.parse_args()
    if not args.ref:
        ap.error("give the reference source tree with --ref or $PHASEFIELD5D_REF")
    gen_configs(args.ref, os.path.join(HERE, "sim_configs.json"))
    if args.only_configs:
        return
    R = import_reference(args.ref)
    gen_save(args.ref, os.path.join(HERE, "save_io.json"))
    if args.only_save:
        return
    table = W.find_unstable_table(small_cfg(2, (12, 10)))[0]
    np.savez_compressed(os.path.join(HERE, "table_small.npz"), data=table.data,
                        resolution=table.resolution, temperature=table.temperature,
                        seed=table.seed)
    gen_kernels(R, table, os.path.join(HERE, "kernels.npz"))
    gen_trajectories(R, table, os.path.join(HERE, "trajectories.npz"))
    with open(os.path.join(HERE, "setup.json"), "w") as f:
        json.dump(gen_setup(R), f, indent=1)
    with open(os.path.join(HERE, "fullres.json"), "w") as f:
        json.dump(gen_fullres(R), f, indent=1)
    print("golden vectors written to", HERE)


if __name__ == "__main__":
    main()
