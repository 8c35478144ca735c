"""Volume preprocessing with the call signatures of pyALDVC's ``al_dvc.io.volume_ops``, computed on the device.

Each function takes a host NumPy volume (and then returns a host array, the reference's contract) or a CUDA
tensor (and then returns a CUDA tensor, the pipeline's fast path):

  normalize_volume   io/volume_ops.py:74-121    (whole volume or a VOI box)
  compute_gradients  io/volume_ops.py:177-197   7-point stencil, zero 3-voxel border
  presmooth_volume   io/volume_ops.py:200-212   Gaussian, edge repeat, per-axis float32 rounding
  prefilter_bspline  io/volume_ops.py:215-222   cubic B-spline coefficients, mirror boundary
  prepare_deformed   io/volume_ops.py:225-244   the array the interpolation samples; masked voxels NaN
"""

from __future__ import annotations

import numpy as np
import torch

from . import kernels as K

GRADIENT_BORDER = 3


def _to_device(vol, dtype=torch.float32):
    if isinstance(vol, torch.Tensor):
        return K.dev(vol, dtype), True
    arr = np.asarray(vol)
    if arr.ndim != 3:
        raise ValueError(f"Expected a 3-D volume, got shape {arr.shape}.")
    return K.dev(np.ascontiguousarray(arr, dtype=np.float32), dtype), False


def _back(t: torch.Tensor, keep_device: bool):
    return t if keep_device else t.cpu().numpy()


def _voi_box(shape, voi):
    """(z0, z1, y0, y1, x0, x1) half-open bounds of the clamped VOI (io/volume_ops.py:40-49); ``voi`` has the
    reference VOIRange's ``clamp(shape).slices``."""
    sz, sy, sx = voi.clamp(tuple(shape)).slices
    z0, z1, _ = sz.indices(shape[0])
    y0, y1, _ = sy.indices(shape[1])
    x0, x1, _ = sx.indices(shape[2])
    if z1 <= z0 or y1 <= y0 or x1 <= x0:
        raise ValueError("VOI is empty after clamping to the volume.")
    return z0, z1, y0, y1, x0, x1


def normalize_volume(vol, voi=None):
    """``(vol - mean) / std`` with the FP64 mean and population std of the (clamped) VOI, or of the whole volume, taken
    relative to the VOI's centre voxel; float32 result, std < 1e-12 taken as 1 (io/volume_ops.py:74-121)."""
    if isinstance(vol, torch.Tensor):
        t = vol.contiguous() if vol.dtype in (torch.float32, torch.uint16) else vol.float().contiguous()
        t = K.dev(t, t.dtype)
        keep = True
    else:
        arr = np.asarray(vol)
        if arr.ndim != 3:
            raise ValueError(f"Expected a 3-D volume, got shape {arr.shape}.")
        t = torch.from_numpy(np.ascontiguousarray(arr if arr.dtype == np.uint16 else arr.astype(np.float32))).cuda()
        keep = False
    if voi is None:
        out = K.normalize(t)
    else:
        out, _ = K.normalize_voi(t, _voi_box(tuple(t.shape), voi))
    return _back(out, keep)


def compute_gradients(f):
    """(gx, gy, gz) of the 7-point central difference, zero within 3 voxels of a face."""
    t, keep = _to_device(f)
    return tuple(_back(g, keep) for g in K.gradients(t, GRADIENT_BORDER))


def presmooth_volume(vol, sigma: float):
    """Gaussian pre-smoothing (``sigma`` in voxels, radius int(4 sigma + 0.5)); identity when ``sigma <= 0``."""
    t, keep = _to_device(vol)
    return _back(K.gaussian_presmooth(t, sigma), keep)


def prefilter_bspline(vol):
    """Cubic B-spline coefficients of ``vol``: sampling them with the cubic B-spline basis reproduces the volume
    at the voxel centres (scipy ``map_coordinates(order=3, mode="mirror")`` between them)."""
    t, keep = _to_device(vol)
    return _back(K.bspline_prefilter(t), keep)


def prepare_deformed(vol, interp_method: str, mask=None):
    """The array the interpolation kernels sample for ``interp_method`` ("linear", "cubic" or "bspline"): the
    B-spline coefficients for "bspline", a float32 copy otherwise; voxels where ``mask`` is False are NaN, so
    any subset voxel whose stencil touches them drops out of that node's correlation."""
    if interp_method not in ("linear", "cubic", "bspline"):
        raise ValueError(f"unknown interp_method {interp_method!r}")
    t, keep = _to_device(vol)
    out = K.bspline_prefilter(t) if interp_method == "bspline" else t.clone()
    if mask is not None:
        m = mask if isinstance(mask, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(np.asarray(mask, dtype=bool)))
        if tuple(m.shape) != tuple(out.shape):
            raise ValueError(f"deformed-frame mask shape {tuple(m.shape)} != volume shape {tuple(out.shape)}")
        K.mask_fill(out, K.dev(m.to(torch.uint8), torch.uint8), float("nan"))
    return _back(out, keep)
