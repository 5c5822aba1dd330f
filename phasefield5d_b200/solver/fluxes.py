"""Kinetic fluxes on the GPU, drop-in for phasefield5d/solver/fluxes.py.

``get_divergence_from_mu_function(dim)`` returns f(X, M, mu, inv_dx, out)
(fluxes.py:398-416): the fused gradient + face-flux + divergence kernel.
``get_flux_function(dim)`` returns f(X, M, gp, gm, fp, fm) (fluxes.py:6-23),
the unfused face fluxes used for save-step diagnostics.
"""
from __future__ import annotations

from .. import _lib
from . import _device as D


def _check_dim(system_dim):
    if system_dim not in (1, 2, 3):
        raise ValueError(f"Unsupported system_dim={system_dim}. Choose 1, 2, or 3.")


def get_divergence_from_mu_function(system_dim):
    _check_dim(system_dim)

    def divergence_from_mu(current_composition, mobilities, mu, inv_dx, out):
        t = D.torch()
        X = D.as_device(current_composition)
        M, ms = D.point_view(mobilities, 5)
        m, mus = D.point_view(mu, 4)
        cuda_out = D.is_cuda_tensor(out) and out.is_contiguous()
        res = out if cuda_out else t.empty_like(X)
        shp, _keep = _lib.shape_arg(X.shape[:-1])
        _lib.check(D.lib().pf5d_divergence_from_mu(
            system_dim, shp, int(X.shape[-1]), _lib.ptr(X), _lib.ptr(M), ms, _lib.ptr(m), mus,
            float(inv_dx), _lib.ptr(res), _lib.stream_handle()), "divergence_from_mu")
        if not cuda_out:
            D.writeback(out, res)
    return divergence_from_mu


def get_flux_function(system_dim):
    _check_dim(system_dim)

    def compute_fluxes(current_composition, mobilities, grad_mu_plus, grad_mu_minus,
                       fluxes_p, fluxes_m):
        X = D.as_device(current_composition)
        M, ms = D.point_view(mobilities, 5)
        gp = D.as_device(grad_mu_plus)
        gm = D.as_device(grad_mu_minus)
        fp = fluxes_p if (D.is_cuda_tensor(fluxes_p) and fluxes_p.is_contiguous()) \
            else D.torch().empty_like(gp)
        fm = fluxes_m if (D.is_cuda_tensor(fluxes_m) and fluxes_m.is_contiguous()) \
            else D.torch().empty_like(gm)
        shp, _keep = _lib.shape_arg(X.shape[:-1])
        _lib.check(D.lib().pf5d_fluxes_pm(system_dim, shp, int(X.shape[-1]), _lib.ptr(X),
                                          _lib.ptr(M), ms, _lib.ptr(gp), _lib.ptr(gm),
                                          _lib.ptr(fp), _lib.ptr(fm), _lib.stream_handle()),
                   "compute_fluxes")
        if fp is not fluxes_p:
            D.writeback(fluxes_p, fp)
        if fm is not fluxes_m:
            D.writeback(fluxes_m, fm)
    return compute_fluxes
