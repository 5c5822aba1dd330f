"""Host-side system helpers for the Cahn-Hilliard step loop: grids, time-step
scalars, Fourier grids, and the linear-stability CTLD setup.

These run once per solve on the host (they size the device buffers and fix the
scalars the device step consumes), so they are plain numpy.  Each function keeps
the name, arguments and arithmetic of the phasefield5d function it stands in
for, so the scalars handed to the device (dx, dt, t_cfl, ctld, B(k)) are the
same numbers the reference main loop would use.

Per-step work (interpolation, stencils, elasticity, reductions, update) never
runs here: it lives in the CUDA library behind ``phasefield5d_b200._lib``.
"""
from __future__ import annotations

import numpy as np


# ---------------------------------------------------------------------------
# Rounding helpers (phasefield5d/utils/statistics.py:44-57)
# ---------------------------------------------------------------------------

def round_to_first_nonzero(x):
    """Round to one significant digit (phasefield5d/utils/statistics.py:44-48)."""
    if x == 0:
        return 0.0
    exponent = int(np.floor(np.log10(abs(x))))
    return round(x, -exponent)


def round_down_to_first_nonzero(x):
    """Truncate to one significant digit (phasefield5d/utils/statistics.py:51-57)."""
    if x == 0:
        return 0.0
    exponent = int(np.floor(np.log10(abs(x))))
    factor = 10 ** exponent
    mantissa = np.floor(abs(x) / factor)
    return np.sign(x) * mantissa * factor


# ---------------------------------------------------------------------------
# Initial condition (phasefield5d/solver/system.py:56-61)
# ---------------------------------------------------------------------------

def apply_fluctuations(reference_composition, size, fluctuation):
    """X = X0 + fluctuation * zero-mean noise, using numpy's *global* RNG.

    Same draw order as phasefield5d/solver/system.py:56-61: one uniform block of
    shape (*size, S+1), centred per point over its S+1 values, first column
    dropped.  Callers seed with ``np.random.seed`` exactly as the reference
    driver does.
    """
    reference_composition = np.asarray(reference_composition, dtype=float)
    num_species = reference_composition.shape[-1]
    base = np.broadcast_to(reference_composition, (*size, num_species))
    noise = (np.random.rand(*size, num_species + 1) - 0.5) * 2.0
    noise -= noise.mean(axis=-1, keepdims=True)
    return base + fluctuation * noise[..., 1:]


# ---------------------------------------------------------------------------
# Time-step scalars (phasefield5d/solver/system.py:80-112)
# ---------------------------------------------------------------------------

def get_time_increment(ctld, steps_per_ctld=100):
    """phasefield5d/solver/system.py:80-81."""
    return round_down_to_first_nonzero(ctld / steps_per_ctld)


def cahn_hilliard_cfl_dt(dx, mobility_max, hessian_max, kappa_max, safety=1):
    """Explicit-Euler stability bound, phasefield5d/solver/system.py:84-87."""
    kmax = np.pi / dx
    dnom = mobility_max * (kappa_max * kmax ** 4 + abs(hessian_max) * kmax ** 2)
    return safety * (2.0 / dnom)


def apply_adaptive_time(dt_current, xdotmax, ctld, t_cfl, *,
                        composition_change_lower_limit=1e-5,
                        composition_change_upper_limit=1e-3,
                        max_change_factor=2.0):
    """Host copy of the adaptive-Δt rule (phasefield5d/solver/system.py:90-112).

    The device step evaluates the same rule in FP64 in a one-block kernel
    after each rate launch (``adaptive_dt`` in csrc/pf5d_device.cuh); this
    host copy serves callers that drive the loop from Python with a host
    ``xdotmax``.
    """
    if xdotmax is None or xdotmax <= 0.0:
        dt_raw = dt_current
    else:
        lo = composition_change_lower_limit / xdotmax
        hi_b = composition_change_upper_limit / xdotmax
        if lo > hi_b:
            lo, hi_b = hi_b, lo
        dt_raw = float(np.clip(dt_current, lo, hi_b))
    hi = dt_current * max_change_factor
    dt_new = min(hi, dt_raw)
    dt_new = min(dt_new, 0.005 * ctld, t_cfl)
    return dt_new


# ---------------------------------------------------------------------------
# System dimensions (phasefield5d/solver/system.py:119-124)
# ---------------------------------------------------------------------------

def get_system_dimensions(wavenumber_max, ppw=16, mw=100, dim=1):
    """(wavelength, cell size, system length, number of cells per axis)."""
    wavelength = 2 * np.pi / wavenumber_max
    target = wavelength / ppw
    system_length = mw * wavelength
    number_of_cells = mw * ppw
    return (wavelength, round_down_to_first_nonzero(target),
            round_to_first_nonzero(system_length), (number_of_cells,) * dim)


# ---------------------------------------------------------------------------
# rfft-compatible Fourier grids (phasefield5d/solver/system.py:140-207)
# ---------------------------------------------------------------------------

def build_fourier_grid_1d_along_direction(n, dx, direction):
    """k-grid of shape (3, n//2+1) along a physical direction (system.py:140-153)."""
    direction = np.asarray(direction, dtype=float)
    direction = direction / np.linalg.norm(direction)
    q = 2.0 * np.pi * np.fft.rfftfreq(n, d=dx)
    k_grid = direction[:, None] * q[None, :]
    k_norm = np.abs(q)
    return k_grid, k_norm


def build_fourier_grid_2d_in_plane(nx, ny, dx, normal):
    """k-grid (3, nx, ny//2+1) in the plane normal to ``normal`` (system.py:156-190).

    In-plane basis by Gram-Schmidt from x (or y when x is nearly parallel to the
    normal), second vector normal × e1.
    """
    normal = np.asarray(normal, dtype=float)
    normal = normal / np.linalg.norm(normal)
    seed_vec = np.array([1.0, 0.0, 0.0])
    if abs(np.dot(seed_vec, normal)) > 0.9:
        seed_vec = np.array([0.0, 1.0, 0.0])
    e1 = seed_vec - np.dot(seed_vec, normal) * normal
    e1 = e1 / np.linalg.norm(e1)
    e2 = np.cross(normal, e1)
    e2 = e2 / np.linalg.norm(e2)
    kx = 2.0 * np.pi * np.fft.fftfreq(nx, d=dx)
    ky = 2.0 * np.pi * np.fft.rfftfreq(ny, d=dx)
    gx, gy = np.meshgrid(kx, ky, indexing="ij")
    k_grid = e1[:, None, None] * gx[None, ...] + e2[:, None, None] * gy[None, ...]
    k_norm = np.sqrt(gx ** 2 + gy ** 2)
    return k_grid, k_norm


def build_fourier_grid_3d(nx, ny, nz, dx):
    """k-grid (3, nx, ny, nz//2+1), rfftfreq on the last axis (system.py:193-207)."""
    kx = 2.0 * np.pi * np.fft.fftfreq(nx, d=dx)
    ky = 2.0 * np.pi * np.fft.fftfreq(ny, d=dx)
    kz = 2.0 * np.pi * np.fft.rfftfreq(nz, d=dx)
    gx, gy, gz = np.meshgrid(kx, ky, kz, indexing="ij")
    k_grid = np.stack([gx, gy, gz], axis=0)
    k_norm = np.linalg.norm(k_grid, axis=0)
    return k_grid, k_norm


def build_fourier_grid_for(dim, shape, dx, direction):
    """Pick the k-grid builder the reference driver uses for ``dim``
    (examples/simulate.py:141-153)."""
    if dim == 1:
        return build_fourier_grid_1d_along_direction(shape[0], dx, direction)
    if dim == 2:
        return build_fourier_grid_2d_in_plane(shape[0], shape[1], dx, direction)
    if dim == 3:
        return build_fourier_grid_3d(shape[0], shape[1], shape[2], dx)
    raise ValueError(f"Unsupported system_dim={dim}. Choose 1, 2, or 3.")


# ---------------------------------------------------------------------------
# Linear-stability analysis (phasefield5d/kinetics/operators.py:8-87)
# ---------------------------------------------------------------------------

def calculate_wavenumber_cutoff(hessian, kappa_matrix):
    """Largest unstable wavenumber k* (kinetics/operators.py:8-18)."""
    import scipy.linalg as la
    if np.all(kappa_matrix == 0):
        lam = np.linalg.eigvalsh(hessian)
    else:
        lam = la.eigvalsh(hessian, kappa_matrix)
    lam_min = lam[0]
    return float(np.sqrt(-lam_min)) if lam_min < 0 else 0.0


def max_growth_rate_scan(hessian, mobility_matrix, kappa_matrix, n_k=10_000):
    """Fastest-growing mode of B(k) = M (H + k² κ) over k in [0.001, 0.999]·k*.

    Same sampling and selection as kinetics/operators.py:21-87 with
    ``max_tag=True``: per k, eigenvalues sorted by real part, growth
    −k²·λ, first strict maximum kept.  Returns (rate, k) or (nan, nan) when
    the composition is stable.  The per-k eigen-solves are batched into one
    ``np.linalg.eig`` call over the stacked operators.
    """
    k_cut = calculate_wavenumber_cutoff(hessian, kappa_matrix)
    if k_cut == 0:
        return np.nan, np.nan
    ks = np.linspace(0.001 * k_cut, 0.999 * k_cut, n_k)
    ops = np.array([mobility_matrix @ (hessian + k ** 2 * kappa_matrix) for k in ks])
    best_rate, best_k = -np.inf, np.nan
    finite = np.isfinite(ops).all(axis=(1, 2))
    vals = np.full((n_k, ops.shape[-1]), np.nan, dtype=complex)
    if finite.any():
        # eig (not eigvals): same LAPACK path per matrix as the reference's
        # per-k np.linalg.eig, so the eigenvalues agree bit for bit.
        vals[finite] = np.linalg.eig(ops[finite])[0]
    for i, k in enumerate(ks):
        if not finite[i]:
            continue
        ev = vals[i][np.argsort(np.real(vals[i]))]
        growth = -(k ** 2) * ev
        j = np.argmax(growth)
        if growth[j] > best_rate:
            best_rate = float(growth[j].real if np.iscomplexobj(growth) else growth[j])
            best_k = k
    if best_rate == -np.inf:
        return np.nan, np.nan
    return best_rate, best_k


def dyadic_mobility_matrix(X0, mob_ref):
    """Dyadic mobility at X0 (phasefield5d/solver/system.py:304-312)."""
    X0 = np.asarray(X0, dtype=float)
    n = X0.shape[0]
    x_fe = 1.0 - X0.sum()
    m_fe = mob_ref[0]
    m_sol = mob_ref[1:]
    v_fe = -X0
    v_sol = np.eye(n) - X0[None, :]
    return (x_fe * m_fe * np.outer(v_fe, v_fe)
            + np.einsum("k,ka,kb->ab", X0 * m_sol, v_sol, v_sol))


def compute_initial_kinetics(initial_composition, resolution, kappa_value, kappa_i,
                             table_eval, elastic_matrix=None, n_k=10_000):
    """CTLD and dominant wavenumber (phasefield5d/solver/system.py:241-329).

    ``table_eval(points) -> (P, 9)`` evaluates the CALPHAD table at host points
    (the reference passes its grid/tree to ``interpolator_nb`` here; the caller
    supplies the equivalent evaluation).  Central differences with
    δ = resolution give the Hessian, the dyadic mobility comes from the table
    at X0, and the kinetic scan picks the fastest-growing mode.

    Raises ``ValueError`` for a composition outside the spinodal, exactly as
    the reference does.
    """
    X0 = np.asarray(initial_composition, dtype=float)
    n = X0.shape[0]
    delta = resolution
    pts = np.vstack([X0[None, :], X0[None, :] + np.eye(n) * delta,
                     X0[None, :] - np.eye(n) * delta])
    vals = table_eval(pts)
    mu_plus = vals[1:n + 1, :n]
    mu_minus = vals[n + 1:, :n]
    mob_ref = vals[0, n:]
    hessian = (mu_plus - mu_minus).T / (2.0 * delta)
    mob = dyadic_mobility_matrix(X0, mob_ref)
    h_total = hessian if elastic_matrix is None else hessian + elastic_matrix
    kappa_mat = np.diag(np.asarray(kappa_i, dtype=float).flatten() * kappa_value)
    rate, kmax = max_growth_rate_scan(h_total, mob, kappa_mat, n_k=n_k)
    if not (rate > 0.0):
        raise ValueError(
            f"No unstable mode found (max_growth_rate={rate:.3e}). "
            "Composition may be outside the spinodal region.")
    return 1.0 / rate, kmax


__all__ = [
    "round_to_first_nonzero", "round_down_to_first_nonzero", "apply_fluctuations",
    "get_time_increment", "cahn_hilliard_cfl_dt", "apply_adaptive_time",
    "get_system_dimensions", "build_fourier_grid_1d_along_direction",
    "build_fourier_grid_2d_in_plane", "build_fourier_grid_3d", "build_fourier_grid_for",
    "calculate_wavenumber_cutoff", "max_growth_rate_scan", "dyadic_mobility_matrix",
    "compute_initial_kinetics",
]
