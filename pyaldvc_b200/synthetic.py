"""Seeded synthetic bead volume pairs with exact ground-truth displacement.

Beads are isotropic Gaussians (peak intensity U(0.5, 1), width ``sigma``) at
uniformly random centres; their number is ``density * n_voxels``.  The
deformed volume re-renders the same beads at ``X_b + u(X_b)`` -- the
Lagrangian convention of the solver (pyALDVC ``synthetic.py:121-137``), but
exact for beads, so no volume resampling error enters the ground truth.

Random streams (``numpy.random.default_rng``): ``seed`` draws the centres and
peaks, ``seed + 1`` the reference noise, ``seed + 2`` the deformed noise.

This NumPy renderer serves volumes up to a few hundred voxels per axis; the
CUDA renderer (``aldvc_render_beads`` in the library) draws the same beads for
the large configurations.
"""

from __future__ import annotations

from dataclasses import dataclass, field
from typing import Callable

import numpy as np

DispFunc = Callable[[np.ndarray, np.ndarray, np.ndarray], tuple[np.ndarray, np.ndarray, np.ndarray]]


def draw_beads(shape, density: float, seed: int):
    """``(centres (B, 3) [z, y, x] float64, peaks (B,) float64)`` for a volume of ``shape``."""
    rng = np.random.default_rng(seed)
    n_beads = int(round(density * float(np.prod(shape))))
    centres = rng.uniform(0.0, 1.0, size=(n_beads, 3)) * np.asarray(shape, dtype=np.float64)[None, :]
    peaks = rng.uniform(0.5, 1.0, size=n_beads)
    return centres, peaks


def render_beads(shape, centres_zyx, peaks, sigma: float, chunk: int = 16384) -> np.ndarray:
    """Sum of Gaussians ``peak * exp(-|x - c|^2 / (2 sigma^2))`` cut at ``ceil(4 sigma)`` voxels."""
    nz, ny, nx = (int(s) for s in shape)
    vol = np.zeros(nz * ny * nx, dtype=np.float64)
    R = int(np.ceil(4.0 * sigma))
    offs = np.arange(-R, R + 1)
    inv = 1.0 / (2.0 * sigma * sigma)
    for s in range(0, centres_zyx.shape[0], chunk):
        c = centres_zyx[s:s + chunk]
        p = peaks[s:s + chunk]
        base = np.floor(c).astype(np.int64)  # (B, 3)
        idx = base[:, :, None] + offs[None, None, :]  # (B, 3, 2R+1)
        w = np.exp(-((idx - c[:, :, None]) ** 2) * inv)  # separable factors
        lim = np.array([nz, ny, nx])[None, :, None]
        inside = (idx >= 0) & (idx < lim)
        w = np.where(inside, w, 0.0)
        idx = np.clip(idx, 0, lim - 1)
        val = p[:, None, None, None] * w[:, 0, :, None, None] * w[:, 1, None, :, None] * w[:, 2, None, None, :]
        flat = (idx[:, 0, :, None, None] * ny + idx[:, 1, None, :, None]) * nx + idx[:, 2, None, None, :]
        vol += np.bincount(flat.ravel(), weights=val.ravel(), minlength=vol.size)
    return vol.reshape(nz, ny, nx).astype(np.float32)


def displace_beads(centres_zyx, disp: DispFunc) -> np.ndarray:
    """Bead centres moved by ``u(X_b)``; ``disp(x, y, z) -> (u, v, w)``."""
    z, y, x = centres_zyx[:, 0], centres_zyx[:, 1], centres_zyx[:, 2]
    u, v, w = disp(x, y, z)
    return np.column_stack([z + w, y + v, x + u])


# --------------------------------------------------------------------------- displacement fields (x, y, z) -> (u, v, w)
def translation(t) -> DispFunc:
    tx, ty, tz = (float(a) for a in t)
    return lambda x, y, z: (np.full_like(x, tx), np.full_like(y, ty), np.full_like(z, tz))


def affine(F, t, centre) -> DispFunc:
    """``u = t + F (x - centre)`` with ``F_ij = du_i/dx_j``."""
    F = np.asarray(F, dtype=np.float64)
    cx, cy, cz = centre
    tx, ty, tz = t

    def fn(x, y, z):
        X, Y, Z = x - cx, y - cy, z - cz
        return (tx + F[0, 0] * X + F[0, 1] * Y + F[0, 2] * Z, ty + F[1, 0] * X + F[1, 1] * Y + F[1, 2] * Z,
                tz + F[2, 0] * X + F[2, 1] * Y + F[2, 2] * Z)

    return fn


def strain_z_plus_sine(eps_z: float, amp: float, period: float, centre) -> DispFunc:
    """Uniaxial strain along z plus ``u_x = amp * sin(2 pi y / period)``."""
    cx, cy, cz = centre

    def fn(x, y, z):
        return amp * np.sin(2.0 * np.pi * y / period), np.zeros_like(y), eps_z * (z - cz)

    return fn


def rotation_z_hydrostatic(angle_deg: float, eps: float, centre) -> DispFunc:
    """Rigid rotation about the z axis through ``centre`` plus hydrostatic strain ``eps``."""
    a = np.deg2rad(angle_deg)
    c, s = np.cos(a), np.sin(a)
    R = np.array([[c, -s, 0.0], [s, c, 0.0], [0.0, 0.0, 1.0]])
    return affine(R - np.eye(3) + eps * np.eye(3), (0.0, 0.0, 0.0), centre)


def indentation(depth_amp: float, a: float, centre_xy, background: float, shape, seed: int) -> DispFunc:
    """Boussinesq-style indentation ``u_z = -depth_amp a^2 / (a^2 + r^2 + d^2)`` (r in-plane radius,
    d depth below z = 0) plus a smooth random-phase background of amplitude ``background`` per component."""
    cx, cy = centre_xy
    nz, ny, nx = shape
    rng = np.random.default_rng(seed)
    ph = rng.uniform(0, 2 * np.pi, size=(3, 3))
    kx, ky, kz = 2 * np.pi / nx, 2 * np.pi / ny, 2 * np.pi / max(nz, 1)

    def bg(x, y, z, c):
        return background / 3.0 * (np.sin(kx * x + ph[c, 0]) + np.sin(ky * y + ph[c, 1]) + np.sin(kz * z + ph[c, 2]))

    def fn(x, y, z):
        r2 = (x - cx) ** 2 + (y - cy) ** 2
        uz = -depth_amp * a * a / (a * a + r2 + z * z)
        return bg(x, y, z, 0), bg(x, y, z, 1), uz + bg(x, y, z, 2)

    return fn


@dataclass
class VolumePair:
    f: np.ndarray
    g: np.ndarray
    disp: DispFunc
    mask: np.ndarray | None = None
    meta: dict = field(default_factory=dict)


def bead_pair(shape, density: float, sigma: float, seed: int, disp: DispFunc, noise: float = 0.01,
              poisson_photons: float | None = None, uint16_max: float | None = None) -> VolumePair:
    """Reference/deformed bead volumes under ``disp``.

    ``noise`` is the Gaussian sigma in units of the bead peak; with ``poisson_photons`` the
    intensities are first Poisson-sampled at that many photons per unit peak.  ``uint16_max``
    rescales to ``[0, uint16_max]`` and rounds to uint16 (both volumes share the scale).
    """
    centres, peaks = draw_beads(shape, density, seed)
    f = render_beads(shape, centres, peaks, sigma)
    g = render_beads(shape, displace_beads(centres, disp), peaks, sigma)
    out = []
    for vol, s in ((f, seed + 1), (g, seed + 2)):
        rng = np.random.default_rng(s)
        v = vol.astype(np.float64)
        if poisson_photons is not None:
            v = rng.poisson(np.maximum(v, 0.0) * poisson_photons) / poisson_photons
        if noise > 0:
            v = v + rng.normal(0.0, noise, size=v.shape)
        out.append(v)
    f64, g64 = out
    if uint16_max is not None:
        lo = min(f64.min(), g64.min())
        hi = max(f64.max(), g64.max())
        scale = uint16_max / max(hi - lo, 1e-12)
        f16 = np.round((f64 - lo) * scale).astype(np.uint16)
        g16 = np.round((g64 - lo) * scale).astype(np.uint16)
        return VolumePair(f16, g16, disp, meta={"scale": scale, "offset": lo})
    return VolumePair(f64.astype(np.float32), g64.astype(np.float32), disp)


def normalize_volume(vol) -> np.ndarray:
    """``(vol - mean) / std`` over the whole volume, FP64 statistics, FP32 result
    (pyALDVC io/volume_ops.normalize_volume :105-121 without a VOI)."""
    a = np.asarray(vol, dtype=np.float64)
    mean = float(a.mean())
    std = float(a.std())
    if std < 1e-12:
        std = 1.0
    return ((a - mean) * (1.0 / std)).astype(np.float32)
