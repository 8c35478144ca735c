"""Per-node displacement uncertainty from the IC-GN normal equations (pyALDVC solver/uncertainty.py).

At a converged node the residual variance per voxel is s^2 = (1 - ZNCC) bottomf^2 / n_valid; the stored Hessian H
carries the reference-gradient noise, E[H] = H0 + c s^2 pattern, with c the variance gain of the 7-point gradient
stencil and pattern the expectation of sum J J^T for unit gradient noise over the subset.  Cov(P) = 2 s^2 H0^-1 +
c s^4 H0^-1 pattern H0^-1; the translation block gives the standard deviation of u, v, w.  The per-node algebra
runs on the device (``aldvc_displacement_uncertainty``); the 12 x 12 pattern of the subset shape is formed here.
"""

from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import kernels as K
from ._lib import check

N_DOF = 12
MIN_EXTRA_DOF = 2  # a node needs n_valid > N_DOF + MIN_EXTRA_DOF voxels for a variance estimate
STENCIL7 = np.array([-1 / 60, 3 / 20, -3 / 4, 0.0, 3 / 4, -3 / 20, 1 / 60], dtype=np.float64)  # io/volume_ops.py:25
STENCIL_NOISE_GAIN = float(np.sum(STENCIL7**2))  # variance gain of the gradient stencil on white noise
MIN_CORRECTED_FRACTION = 0.1  # the correction keeps at least this fraction of each translation diagonal


def subset_moment_matrix(half, stride: int = 1) -> np.ndarray:
    """diag(sum X^2, sum Y^2, sum Z^2, n) over the sampled subset (uncertainty.py:47-59; the cross moments vanish
    on the symmetric subset)."""
    hx, hy, hz = (int(h) for h in half)
    ax, ay, az = (np.arange(-h, h + 1, int(stride)) for h in (hx, hy, hz))
    nx, ny, nz = ax.size, ay.size, az.size
    return np.diag([float(np.sum(ax**2)) * ny * nz, float(np.sum(ay**2)) * nx * nz, float(np.sum(az**2)) * nx * ny,
                    float(nx * ny * nz)])


def noise_hessian_pattern(half, stride: int = 1) -> np.ndarray:
    """(12, 12): E[sum J J^T]_pq = [component(p) == component(q)] M[coordinate(p), coordinate(q)] for P = [F, u, v, w]
    (F row-major: parameter p < 9 is gradient component p // 3 times coordinate p % 3; u, v, w times 1)."""
    M = subset_moment_matrix(half, stride)
    comp = np.array([p // 3 for p in range(9)] + [0, 1, 2])
    coord = np.array([p % 3 for p in range(9)] + [3, 3, 3])
    return np.where(comp[:, None] == comp[None, :], M[coord[:, None], coord[None, :]], 0.0)


def displacement_uncertainty_device(H: torch.Tensor, zncc: torch.Tensor, status: torch.Tensor | None, valid: torch.Tensor,
                                    n_valid: torch.Tensor, bottomf: torch.Tensor, half, stride: int = 1,
                                    noise_correction: bool = True) -> torch.Tensor:
    """(N, 3) FP64 standard deviation of u, v, w (voxels), NaN where undefined (uncertainty.py:94-137)."""
    pattern = np.ascontiguousarray(noise_hessian_pattern(half, stride), dtype=np.float64)
    N = int(zncc.shape[0])
    out = torch.empty((N, 3), dtype=torch.float64, device=zncc.device)
    args = [K.dev(H, torch.float64), K.dev(zncc, torch.float64), None if status is None else K.dev(status, torch.int8),
            K.dev(valid, torch.uint8), K.dev(n_valid, torch.int64), K.dev(bottomf, torch.float64)]
    check(K.lib().aldvc_displacement_uncertainty(*[K._p(a) for a in args], N, pattern.ctypes.data_as(ctypes.c_void_p),
                                                 STENCIL_NOISE_GAIN, MIN_CORRECTED_FRACTION, int(bool(noise_correction)), K._p(out),
                                                 K.stream_handle()), "aldvc_displacement_uncertainty")
    return out
