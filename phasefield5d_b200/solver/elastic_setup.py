"""Host-side construction of the Khachaturyan elastic operator.

Builds, once per solve, what the device elastic step consumes:

* the real Fourier-space kernel B(k) on the rfft half-grid
  (phasefield5d/solver/elastic.py:73-107),
* the scalar anisotropy B(n) for one direction, used in the CTLD Hessian
  (phasefield5d/elasticity/anisotropy.py:35-65, solver/elastic.py:61-66),
* the rank-1 factor l with Λ = l lᵀ (phasefield5d/solver/elastic.py:190-197).

The per-step elastic update itself (misfit contraction, B(k) multiply, rank-1
expansion around one cuFFT pair) runs on the GPU; see ``elastic.py``.
"""
from __future__ import annotations

import numpy as np


def _phi_terms(c11, c12, c44):
    a = c11 - c12 - 2.0 * c44
    b = c11 + c12 + 2.0 * c44
    d = c11 + 2.0 * c12 + 4.0 * c44
    return a, b, d


def khachaturyan_anisotropy(n, c11, c12, c44):
    """(B_n, Y_n) in GPa for one direction n (elasticity/anisotropy.py:35-65)."""
    n1, n2, n3 = np.asarray(n, dtype=float) / np.linalg.norm(n)
    a, b, d = _phi_terms(c11, c12, c44)
    nf1 = n1 ** 2 * n2 ** 2 + n2 ** 2 * n3 ** 2 + n3 ** 2 * n1 ** 2
    nf2 = n1 ** 2 * n2 ** 2 * n3 ** 2
    phi = c11 * (1 + 2 * a / c44 * nf1 + 3 * (a / c44) ** 2 * nf2) / (
        c11 + a * (c11 + c12) / c44 * nf1 + (a / c44) ** 2 * b * nf2)
    phi_avg = 1 + 4 * a / b / 5 + 54 * a ** 2 / (b * d) / 105
    prefac = (c11 + 2 * c12) ** 2 / c11
    return -prefac * (phi - phi_avg), 3 * (c11 + 2 * c12) - prefac * phi


def build_khachaturyan_kernel(k_grid, k_norm, c11, c12, c44):
    """B(k) in J/m³ on a k-grid; B = 0 at k = 0 (solver/elastic.py:73-107)."""
    nonzero = k_norm > 0.0
    with np.errstate(invalid="ignore", divide="ignore"):
        n1 = np.where(nonzero, k_grid[0] / k_norm, 0.0)
        n2 = np.where(nonzero, k_grid[1] / k_norm, 0.0)
        n3 = np.where(nonzero, k_grid[2] / k_norm, 0.0)
    a, b, d = _phi_terms(c11, c12, c44)
    nf1 = n1 ** 2 * n2 ** 2 + n2 ** 2 * n3 ** 2 + n3 ** 2 * n1 ** 2
    nf2 = n1 ** 2 * n2 ** 2 * n3 ** 2
    phi = np.where(
        nonzero,
        c11 * (1.0 + 2.0 * a / c44 * nf1 + 3.0 * (a / c44) ** 2 * nf2)
        / (c11 + a * (c11 + c12) / c44 * nf1 + (a / c44) ** 2 * b * nf2),
        1.0,
    )
    phi_avg = 1.0 + 4.0 * a / b / 5.0 + 54.0 * a ** 2 / (b * d) / 105.0
    b_n = np.where(nonzero, -(c11 + 2.0 * c12) ** 2 / c11 * (phi - phi_avg), 0.0)
    return b_n * 1e9


def calculate_molar_volume(X, Vi):
    """Linear-mixing molar volume (elasticity/energies.py:18-26)."""
    X = np.asarray(X, dtype=float)
    return Vi[0] * (1.0 - np.sum(X)) + np.dot(Vi[1:], X)


def coupling_matrix(misfit):
    """Λ = l lᵀ from Vegard misfit coefficients (solver/elastic.py:55-58)."""
    misfit = np.asarray(misfit, dtype=float)
    return np.outer(misfit, misfit)


def get_elastic_matrix(misfit, molar_volume, c11, c12, c44, direction=(1, 0, 0)):
    """Λ · B_n · 1e9 · V_m in J/mol: the elastic term of the CTLD Hessian
    (solver/elastic.py:61-66, with the misfit supplied directly)."""
    b_n, _ = khachaturyan_anisotropy(np.asarray(direction), c11, c12, c44)
    return coupling_matrix(misfit) * b_n * 1e9 * molar_volume


def rank1_factor(linear_elastic_coupling_matrix, dtype=np.float64):
    """Return l with Λ = l lᵀ, or None when Λ is not rank 1 (elastic.py:190-197).

    Uses the same symmetric eigen-decomposition as the reference so the
    factor (and its arbitrary sign) is the same vector the CPU path uses.
    """
    eigvals, eigvecs = np.linalg.eigh(linear_elastic_coupling_matrix)
    largest = eigvals[-1]
    n_nonzero = int(np.sum(eigvals > 1e-10 * max(largest, 1e-30)))
    if n_nonzero == 1 and largest > 0.0:
        return (eigvecs[:, -1] * np.sqrt(largest)).astype(dtype)
    return None


def k_shape_for(spatial_shape):
    """rfft half-grid shape for a real field (solver/elastic.py:169-177)."""
    if len(spatial_shape) == 1:
        return (spatial_shape[0] // 2 + 1,)
    if len(spatial_shape) == 2:
        return (spatial_shape[0], spatial_shape[1] // 2 + 1)
    if len(spatial_shape) == 3:
        return (spatial_shape[0], spatial_shape[1], spatial_shape[2] // 2 + 1)
    raise NotImplementedError(
        f"make_elastic_updater not implemented for spatial_dim={len(spatial_shape)}")
