"""Uniform hex8 node grid (the caller side of the solver boundary).

Same placement rule and node numbering as pyALDVC ``mesh/grid_mesh.py``:
nodes keep ``GRADIENT_BORDER + INTERP_MARGIN`` voxels plus half a subset
away from every face, are centred in the available span
(``build_grid_axes`` :19-60), node ``n = iz*ny*nx + iy*nx + ix`` with
coordinates ``[x, y, z]`` and hex8 corner order n0..n7 (``mesh_setup``
:63-122).
"""

from __future__ import annotations

import numpy as np

GRADIENT_BORDER = 3
INTERP_MARGIN = 2


def build_grid_axes(volume_shape, winsize, winstepsize, voi=None, extra_margin: int = 0):
    """Node axes ``(x0, y0, z0)``; ``voi`` is ``((xlo, xhi), (ylo, yhi), (zlo, zhi))`` inclusive or None."""
    nz, ny, nx = volume_shape
    if voi is None:
        voi = ((0, nx - 1), (0, ny - 1), (0, nz - 1))
    axes = []
    for axis_len, (lo, hi), w, h in zip((nx, ny, nz), voi, winsize, winstepsize):
        half = int(w) // 2
        border = GRADIENT_BORDER + INTERP_MARGIN + int(extra_margin)
        first = max(lo, border) + half
        last = min(hi, axis_len - 1 - border) - half
        if last < first:
            raise ValueError(f"subset {w} does not fit in ({lo}, {hi}) of a {axis_len}-voxel axis")
        n = int((last - first) // h) + 1
        if n < 2:
            raise ValueError("fewer than 2 nodes along an axis")
        span = (n - 1) * h
        start = first + (last - first - span) // 2
        axes.append(np.arange(n, dtype=np.float64) * h + start)
    return axes[0], axes[1], axes[2]


def grid_coords(x0, y0, z0) -> np.ndarray:
    """``(N, 3)`` [x, y, z] node coordinates, x fastest."""
    Z, Y, X = np.meshgrid(z0, y0, x0, indexing="ij")
    return np.column_stack([X.ravel(), Y.ravel(), Z.ravel()])


def grid_elements(grid_shape) -> np.ndarray:
    """``(E, 8)`` hex8 connectivity of the full grid (element ``e = ez*(ny-1)*(nx-1) + ey*(nx-1) + ex``)."""
    nz, ny, nx = grid_shape
    iz, iy, ix = (a.ravel() for a in np.meshgrid(np.arange(nz - 1), np.arange(ny - 1), np.arange(nx - 1), indexing="ij"))

    def nid(a, b, c):
        return c * ny * nx + b * nx + a

    return np.column_stack([nid(ix, iy, iz), nid(ix + 1, iy, iz), nid(ix + 1, iy + 1, iz), nid(ix, iy + 1, iz),
                            nid(ix, iy, iz + 1), nid(ix + 1, iy, iz + 1), nid(ix + 1, iy + 1, iz + 1),
                            nid(ix, iy + 1, iz + 1)]).astype(np.int64)


def element_active(grid_shape, node_valid) -> np.ndarray:
    """Elements whose 8 corners are valid nodes (pyALDVC ``apply_mask_to_mesh`` :219-222)."""
    v = np.asarray(node_valid, dtype=bool).ravel()
    return v[grid_elements(grid_shape)].all(axis=1)


def surface_nodes(grid_shape) -> np.ndarray:
    """Nodes on the outer surface of the grid (``grid_surface_nodes`` :125-132)."""
    on = np.zeros(grid_shape, dtype=bool)
    on[0], on[-1] = True, True
    on[:, 0], on[:, -1] = True, True
    on[:, :, 0], on[:, :, -1] = True, True
    return np.flatnonzero(on.ravel())
