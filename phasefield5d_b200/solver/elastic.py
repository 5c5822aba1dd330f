"""Khachaturyan elasticity: host construction plus the GPU per-step update,
drop-in for phasefield5d/solver/elastic.py.

``make_elastic_updater`` keeps the reference signature and returns
``elastic_update(mu, X)``.  For the rank-1 coupling matrix (always the case
for Vegard misfits) the update runs as one cuFFT D2Z/Z2D pair with the
misfit contraction, B(k) multiply and rank-1 expansion as hand-written
kernels (``pf5d_elastic_*``).  A non-rank-1 matrix is rejected: the GPU path
implements the reference's rank-1 branch only.
"""
from __future__ import annotations

import ctypes

import numpy as np

from .. import _lib
from . import _device as D
from .elastic_setup import (build_khachaturyan_kernel, calculate_molar_volume,  # noqa: F401
                            coupling_matrix, get_elastic_matrix, k_shape_for,
                            khachaturyan_anisotropy, rank1_factor)


def calculate_linear_elastic_coupling_matrix(misfit):
    """Λ = l lᵀ (solver/elastic.py:55-58), from the misfit coefficients."""
    return coupling_matrix(misfit)


class _ElasticHandle:
    def __init__(self, dim, shape, x0, lvec, bk):
        L = D.lib()
        shp, self._keep = _lib.shape_arg(shape)
        x0p, k1 = _lib.f64_array(x0)
        lp, k2 = _lib.f64_array(lvec)
        bk = np.ascontiguousarray(bk, dtype=np.float64)
        h = ctypes.c_void_p()
        _lib.check(L.pf5d_elastic_create(dim, shp, x0p, lp,
                                         bk.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                         ctypes.byref(h)), "make_elastic_updater")
        self.h = h
        self._lib = L

    def __del__(self):
        try:
            if self.h:
                self._lib.pf5d_elastic_destroy(self.h)
        except Exception:
            pass


def make_elastic_updater(cfg, linear_elastic_coupling_matrix, elastic_kernel_r, field_shape,
                         field_dtype=np.float64, fft_workers=1):
    """solver/elastic.py:147-286 (rank-1 path) on the device."""
    if not getattr(cfg, "include_cubic_anisotropy", True) or elastic_kernel_r is None:
        def elastic_update(mu, X):
            return
        return elastic_update
    spatial = tuple(field_shape[:-1])
    k_shape = k_shape_for(spatial)
    if tuple(np.shape(elastic_kernel_r)) != k_shape:
        raise AssertionError(f"elastic_kernel_r shape {np.shape(elastic_kernel_r)} does not "
                             f"match expected {k_shape}")
    lvec = rank1_factor(np.asarray(linear_elastic_coupling_matrix, dtype=np.float64))
    if lvec is None:
        raise NotImplementedError("the GPU elastic update implements the rank-1 coupling path")
    x0 = np.asarray(cfg.initial_composition, dtype=np.float64)
    handle = _ElasticHandle(len(spatial), spatial, x0, lvec, np.asarray(elastic_kernel_r))

    def elastic_update(chemical_potentials, composition_field):
        X = D.as_device(composition_field)
        mu, mus = D.point_view(chemical_potentials, 4)
        _lib.check(handle._lib.pf5d_elastic_apply(handle.h, _lib.ptr(mu), mus, _lib.ptr(X),
                                                  _lib.stream_handle()), "elastic_update")
        if not D.is_cuda_tensor(chemical_potentials):
            D.writeback(chemical_potentials, mu)
    elastic_update.lvec = lvec
    elastic_update.handle = handle
    return elastic_update
