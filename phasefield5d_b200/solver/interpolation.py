"""4D CALPHAD interpolation on the GPU, drop-in for
phasefield5d/solver/interpolation.py.

``interpolator_nb`` keeps the reference signature.  The table evaluation and
the nearest-row fallback both run on the device (``pf5d_interp4d``); the
``tree`` argument supplies the row compositions for the fallback's distance
test (the device searches the dense grid's present nodes, which are exactly
the table rows), ``calphad_values`` is accepted for signature compatibility.
"""
from __future__ import annotations

import ctypes

import numpy as np

from .. import _lib
from . import _device as D
from .table import build_4d_grid, build_calphad_kdtree  # noqa: F401  (reference names)


def interpolator_nb(composition_array, data_grid, resolution, tree, calphad_values,
                    max_nn_dist=None, out=None, mask_buffer=None):
    """phasefield5d/solver/interpolation.py:154-211 on the device.

    Accepts numpy arrays (copied to the device, results copied back into
    ``out`` / ``mask_buffer``) or CUDA tensors (used in place).  The
    fallback row is the exact nearest table row for any finite point, on or
    off the simplex.  Raises where the reference raises: ``RuntimeError``
    when ``max_nn_dist`` is set and a fallback row is farther than it, and
    ``ValueError`` for a non-finite composition that takes the fallback
    (``cKDTree.query`` rejects it).
    """
    t = D.torch()
    L = D.lib()
    comp = D.as_device(composition_array)
    sp = tuple(comp.shape[:-1])
    n_props = int(data_grid.shape[4])
    npts = int(np.prod(sp)) if sp else 1
    grid, coord = D.TABLES.get(data_grid, resolution, tree)
    if out is None:
        res = t.empty((*sp, n_props), dtype=t.float64, device="cuda")
        host_out = not D.is_cuda_tensor(composition_array)
    else:
        res = out if D.is_cuda_tensor(out) else t.empty((*sp, n_props), dtype=t.float64,
                                                       device="cuda")
        host_out = False
    mask = t.empty(npts, dtype=t.uint8, device="cuda")
    flags = t.zeros(1, dtype=t.int32, device="cuda")
    _lib.check(L.pf5d_interp4d(_lib.ptr(comp), npts, _lib.ptr(grid), int(data_grid.shape[0]),
                               n_props, int(grid.shape[-1]), float(resolution), _lib.ptr(coord),
                               float(max_nn_dist) if max_nn_dist is not None else -1.0,
                               _lib.ptr(res), n_props, _lib.ptr(mask), _lib.ptr(flags),
                               _lib.stream_handle()), "interpolator_nb")
    _lib.raise_nn_errors(int(flags.item()), check_far=max_nn_dist is not None)
    if mask_buffer is not None:
        if D.is_cuda_tensor(mask_buffer):
            mask_buffer.copy_(mask.view(mask_buffer.shape).to(mask_buffer.dtype))
        else:
            mask_buffer[...] = mask.cpu().numpy().astype(bool).reshape(mask_buffer.shape)
    if out is not None and not D.is_cuda_tensor(out):
        return D.writeback(out, res)
    if host_out:
        return res.cpu().numpy()
    return res


__all__ = ["interpolator_nb", "build_4d_grid", "build_calphad_kdtree", "ctypes"]
