"""Array plumbing for the drop-in functions: numpy arrays are copied to the
device and results copied back into the caller's arrays; CUDA torch tensors
are used in place.  Every compute call goes to libpf5d.so."""
from __future__ import annotations

import weakref

import numpy as np

from .. import _lib


def torch():
    import torch as _t
    return _t


def is_cuda_tensor(a):
    t = torch()
    return isinstance(a, t.Tensor) and a.is_cuda


def as_device(a, dtype=None, contiguous=True):
    """CUDA float64 tensor view/copy of ``a`` (numpy array or tensor)."""
    t = torch()
    dtype = dtype or t.float64
    if isinstance(a, t.Tensor):
        x = a.to(device="cuda", dtype=dtype)
    else:
        x = t.from_numpy(np.ascontiguousarray(np.asarray(a, dtype=np.float64))).to("cuda")
        if dtype != t.float64:
            x = x.to(dtype)
    if contiguous and not x.is_contiguous():
        x = x.contiguous()
    return x


def writeback(dst, src):
    """Copy device result ``src`` into caller array ``dst`` (numpy or tensor)."""
    t = torch()
    if isinstance(dst, t.Tensor):
        if dst.data_ptr() != src.data_ptr():
            dst.copy_(src.view(dst.shape))
    else:
        dst[...] = src.view(dst.shape).cpu().numpy()
    return dst


def point_view(a, ncomp):
    """(tensor, point_stride) for a (*sp, C) array whose last axis is unit
    stride (views such as interp[..., :4] keep their stride)."""
    t = torch()
    if isinstance(a, t.Tensor) and a.is_cuda and a.dtype == t.float64 and a.stride(-1) == 1:
        sp = a.shape[:-1]
        strides = a.stride()[:-1]
        # the point index must map to a constant stride (C-ordered views)
        expect = a.stride(-2) if a.dim() >= 2 else a.shape[-1]
        ok = all(strides[i] == expect * int(np.prod(sp[i + 1:])) for i in range(len(sp)))
        if ok:
            return a, expect
    x = as_device(a)
    return x, ncomp


class DeviceTableCache:
    """Device copy of a host table, keyed by the host array's identity."""

    def __init__(self):
        self._entries = {}

    def get(self, data_grid, resolution, tree):
        from .table import node_coordinates
        t = torch()
        if isinstance(data_grid, t.Tensor) and data_grid.is_cuda:
            key = ("t", data_grid.data_ptr(), tuple(data_grid.shape), id(tree))
            ent = self._entries.get(key)
            if ent is None:
                coord = t.from_numpy(node_coordinates(tree, resolution)).to("cuda")
                ent = (None, data_grid.contiguous(), coord)
                self._entries[key] = ent
            return ent[1], ent[2]
        key = ("n", id(data_grid), id(tree), float(resolution))
        ent = self._entries.get(key)
        if ent is not None and ent[0]() is data_grid:
            return ent[1], ent[2]
        grid = t.from_numpy(np.ascontiguousarray(data_grid, dtype=np.float64)).to("cuda")
        coord = t.from_numpy(node_coordinates(tree, resolution)).to("cuda")
        try:
            ref = weakref.ref(data_grid)
        except TypeError:
            ref = (lambda obj: (lambda: obj))(data_grid)
        self._entries[key] = (ref, grid, coord)
        return grid, coord


TABLES = DeviceTableCache()


def lib():
    return _lib.load()
