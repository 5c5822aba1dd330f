"""CALPHAD table containers: dense 4D grid and node set.

``build_4d_grid`` and ``build_calphad_kdtree`` keep the reference's arguments
and outputs (phasefield5d/solver/interpolation.py:13-44): a dense
``(n, n, n, n, n_props)`` grid holding each table row at its composition node
(NaN elsewhere), and a KD-tree over the row compositions with the row values.

``DeviceTable`` is the device-resident form used by every GPU entry point: the
dense grid in HBM (props innermost, so the two nodes along the last axis are
one 144-byte run for 9 FP64 props), plus the per-axis node coordinates used by
the on-device nearest-node fallback.

``host_table_eval`` evaluates the table on a handful of host points for setup
(the CTLD finite-difference stencil and the reference point X0); it is not on
the step path.
"""
from __future__ import annotations

import numpy as np


def build_4d_grid(original_data, resolution, dtype=np.float64):
    """(xdim, grid): rows of [x1..x4, props...] placed on a dense 4D grid.

    Node index = rint(x / resolution), clipped to [0, n-1]; unfilled nodes are
    NaN (phasefield5d/solver/interpolation.py:13-35).
    """
    data = original_data.to_numpy() if hasattr(original_data, "to_numpy") else np.asarray(original_data)
    n_props = data[:, 4:].shape[-1]
    step = float(resolution)
    num = int(round(1.0 / step)) + 1
    xdim = np.linspace(0.0, 1.0, num)
    coords = data[:, :4].astype(np.float64, copy=False)
    values = data[:, 4:4 + n_props].astype(dtype, copy=False)
    idx = np.clip(np.rint(coords / step).astype(np.int32), 0, num - 1)
    grid = np.full((num, num, num, num, n_props), np.nan, dtype=dtype)
    grid[idx[:, 0], idx[:, 1], idx[:, 2], idx[:, 3], :] = values
    return xdim, grid


def build_calphad_kdtree(original_data):
    """(cKDTree over row compositions, row values) (interpolation.py:38-44)."""
    from scipy.spatial import cKDTree
    data = (original_data.to_numpy() if hasattr(original_data, "to_numpy")
            else np.asarray(original_data, dtype=float))
    return cKDTree(data[:, :4].astype(float)), data[:, 4:].astype(float)


def node_coordinates(tree_or_coords, resolution):
    """Per-axis coordinate of each node index, as stored in the table rows.

    The device nearest-node search measures distances to the row
    compositions, so it needs the exact stored coordinate of node k along an
    axis (e.g. the double nearest 0.075, not 3*0.025).  Rows lie on a
    tensor grid, so one table of n values serves all four axes; this is
    checked here.
    """
    coords = getattr(tree_or_coords, "data", tree_or_coords)
    coords = np.asarray(coords, dtype=np.float64)
    num = int(round(1.0 / float(resolution))) + 1
    axis = np.full(num, np.nan)
    idx = np.clip(np.rint(coords / resolution).astype(np.int64), 0, num - 1)
    for d in range(4):
        axis[idx[:, d]] = coords[:, d]
    for d in range(4):
        if not np.array_equal(axis[idx[:, d]], coords[:, d]):
            raise ValueError("table rows are not on one tensor grid; "
                             "the device nearest-node search needs shared axis coordinates")
    missing = np.isnan(axis)
    if missing.any():
        k = np.arange(num)[missing]
        axis[missing] = k * float(resolution)
    return axis


class DeviceTable:
    """Dense table + node coordinates resident on one CUDA device.

    ``grid`` is (n, n, n, n, n_props) contiguous in the requested dtype; the
    ``mu_shift`` (FP32 form only) is subtracted from the μ columns before the
    cast so FP32 stores the small deviation μ − μ(X0) instead of μ.
    """

    def __init__(self, grid, resolution, node_coord, device="cuda", dtype=None,
                 mu_shift=None):
        import torch
        grid = np.asarray(grid)
        self.n = int(grid.shape[0])
        self.n_props = int(grid.shape[-1])
        self.resolution = float(resolution)
        host = grid.astype(np.float64, copy=True)
        if mu_shift is not None:
            host[..., :len(mu_shift)] -= np.asarray(mu_shift, dtype=np.float64)
        tdtype = torch.float64 if dtype in (None, np.float64, "float64") else torch.float32
        self.grid = torch.from_numpy(np.ascontiguousarray(host)).to(device=device, dtype=tdtype)
        self.node_coord = torch.from_numpy(np.ascontiguousarray(node_coord, dtype=np.float64)).to(device)
        self.mu_shift = None if mu_shift is None else np.asarray(mu_shift, dtype=np.float64)


def host_table_eval(points, grid, resolution, tree=None, values=None):
    """Quadrilinear table evaluation on a few host points (setup only).

    Same clamp/weight/summation order as the device kernel; rows outside the
    linear region (Σx > 1 − 4·res − 1e-9) take the nearest table row.
    """
    pts = np.atleast_2d(np.asarray(points, dtype=np.float64))
    num = grid.shape[0]
    n_props = grid.shape[-1]
    inv = 1.0 / resolution
    thr = 1.0 - 4.0 * resolution - 1e-9
    out = np.empty((pts.shape[0], n_props))
    for r, x in enumerate(pts):
        s = 0.0
        for d in range(4):
            s += x[d]
        if not s <= thr:
            if tree is None:
                raise ValueError("point outside the linear region and no tree given")
            _, j = tree.query(x)
            out[r] = values[j]
            continue
        ii, tt = [], []
        for d in range(4):
            u = x[d] * inv
            if u <= 0.0:
                i, t = 0, 0.0
            elif u >= num - 1:
                i, t = num - 2, 1.0
            else:
                i = int(u)
                t = u - i
            ii.append(i)
            tt.append(t)
        ss = [1.0 - t for t in tt]
        acc = np.zeros(n_props)
        first = True
        for b0 in (0, 1):
            for b1 in (0, 1):
                for b2 in (0, 1):
                    for b3 in (0, 1):
                        w = ((tt[0] if b0 else ss[0]) * (tt[1] if b1 else ss[1])
                             * (tt[2] if b2 else ss[2]) * (tt[3] if b3 else ss[3]))
                        term = w * grid[ii[0] + b0, ii[1] + b1, ii[2] + b2, ii[3] + b3, :]
                        acc = term if first else acc + term
                        first = False
        out[r] = acc
    return out
