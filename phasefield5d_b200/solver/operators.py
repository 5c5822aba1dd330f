"""Stencil operators and reductions on the GPU, drop-in for
phasefield5d/solver/operators.py (calculate_laplacian, calculate_gradients_pm,
abs_max, clamp_simplex)."""
from __future__ import annotations

import numpy as np

from .. import _lib
from . import _device as D


def calculate_laplacian(array, cell_size, out=None):
    """operators.py:10-29: periodic second-order Laplacian, same shape."""
    t = D.torch()
    c = D.as_device(array)
    dim = c.dim() - 1
    if dim not in (1, 2, 3):
        raise NotImplementedError(f"Laplacian not implemented for spatial_dims={dim}")
    res = out if (out is not None and D.is_cuda_tensor(out) and out.is_contiguous()) \
        else t.empty_like(c)
    shp, _keep = _lib.shape_arg(c.shape[:-1])
    _lib.check(D.lib().pf5d_laplacian(dim, shp, int(c.shape[-1]), _lib.ptr(c), float(cell_size),
                                      _lib.ptr(res), _lib.stream_handle()), "calculate_laplacian")
    if out is not None and not (D.is_cuda_tensor(out) and out.is_contiguous()):
        return D.writeback(out, res)
    return res if D.is_cuda_tensor(array) else res.cpu().numpy()


def calculate_gradients_pm(array, cell_size, grad_p=None, grad_m=None):
    """operators.py:79-123: forward/backward gradients, (dim, *sp, C) each."""
    t = D.torch()
    ncomp = int(array.shape[-1])
    c, cs = D.point_view(array, ncomp)
    dim = c.dim() - 1
    if dim not in (1, 2, 3):
        raise NotImplementedError(f"Gradients not implemented for spatial_dims={dim}")
    sp = tuple(c.shape[:-1])
    gp = t.empty((dim, *sp, ncomp), dtype=t.float64, device="cuda")
    gm = t.empty_like(gp)
    shp, _keep = _lib.shape_arg(sp)
    _lib.check(D.lib().pf5d_gradients_pm(dim, shp, ncomp, _lib.ptr(c), cs, float(cell_size),
                                         _lib.ptr(gp), _lib.ptr(gm), _lib.stream_handle()),
               "calculate_gradients_pm")
    if D.is_cuda_tensor(array):
        if grad_p is not None:
            grad_p.copy_(gp)
            gp = grad_p
        if grad_m is not None:
            grad_m.copy_(gm)
            gm = grad_m
        return gp, gm
    gp_h, gm_h = gp.cpu().numpy(), gm.cpu().numpy()
    if grad_p is not None:
        grad_p[...] = gp_h
        gp_h = grad_p
    if grad_m is not None:
        grad_m[...] = gm_h
        gm_h = grad_m
    return gp_h, gm_h


def abs_max(arr):
    """operators.py:161-175: max |a| over all elements (NaN ignored), as float."""
    t = D.torch()
    a = D.as_device(arr)
    res = t.empty(1, dtype=t.float64, device="cuda")
    _lib.check(D.lib().pf5d_abs_max(_lib.ptr(a), int(a.numel()), _lib.ptr(res),
                                    _lib.stream_handle()), "abs_max")
    return float(res.item())


def clamp_simplex(composition):
    """operators.py:304-317: renormalise points with sum > 1, in place."""
    dim = composition.ndim - 1 if hasattr(composition, "ndim") else composition.dim() - 1
    if dim not in (1, 2, 3):
        raise NotImplementedError(f"clamp_simplex not implemented for spatial_dims={dim}")
    x = D.as_device(composition)
    ncomp = int(x.shape[-1])
    _lib.check(D.lib().pf5d_clamp_simplex(_lib.ptr(x), int(x.numel() // ncomp), ncomp,
                                          _lib.stream_handle()), "clamp_simplex")
    D.writeback(composition, x)


def out_of_bounds(composition, tol_soft=1e-5, tol_hard=1e-3):
    """phasefield5d/solver/system.py:12-53 with the statistics reduced on the
    device.  Prints the reference's messages; returns True for hard violations."""
    x = D.as_device(composition)
    ncomp = int(x.shape[-1])
    ptr, keep = _lib.f64_array([0.0] * 5)
    _lib.check(D.lib().pf5d_oob_stats(_lib.ptr(x), int(x.numel() // ncomp), ncomp, ptr,
                                      _lib.stream_handle()), "out_of_bounds")
    n_bad, sums_max, sums_min, comp_max, comp_min = list(keep)
    if n_bad > 0:
        print("HARD OUT OF BOUNDS: non-finite value (NaN/inf) present")
        return True
    soft, hard = [], []
    checks = [(sums_max > 1.0 + tol_soft, sums_max > 1.0 + tol_hard,
               f"sum(N-1) > 1 + tol. max sum={sums_max:.8f}"),
              (sums_min < 0.0 - tol_soft, sums_min < 0.0 - tol_hard,
               f"sum(N-1) < -tol. min sum={sums_min:.8f}"),
              (comp_min < 0.0 - tol_soft, comp_min < 0.0 - tol_hard,
               f"component < -tol. min comp={comp_min:.8f}"),
              (comp_max > 1.0 + tol_soft, comp_max > 1.0 + tol_hard,
               f"component > 1 + tol. max comp={comp_max:.8f}")]
    for is_soft, is_hard, text in checks:
        if is_soft:
            soft.append("SOFT OOB: " + text)
        if is_hard:
            hard.append("HARD OOB: " + text)
    for m in soft:
        print(m)
    for m in hard:
        print(m)
    return bool(hard)


__all__ = ["calculate_laplacian", "calculate_gradients_pm", "abs_max", "clamp_simplex",
           "out_of_bounds", "np"]
