"""Seeded inputs of golden_pass.npz (whole AL-DVC passes of the reference's run_aldvc) and of
golden_ncc_fft.npz (integer searches on the reference's FFT branch), shared by make_golden.py, which feeds
them to the reference, and the tests, which regenerate them instead of storing the volumes and check their
SHA-256 against the fixtures.

Pass cases (dict of the reference's DVCPara fields beside the volume recipe):
  affine  56 x 64 x 72 float32 beads, affine field; ws 16 / step 8, direct NCC +-4, tricubic, ADMM with the
          reference's early stop;
  masked  the same pair with a spherical reference mask (nodes and elements dropped), trilinear, three ADMM
          steps (admm_tol 0);
  fft     80 x 80 x 88 uint16 (0-4095) beads, sigma 2, Poisson (1000 photons per unit peak) plus Gaussian noise; ws 32 / step 12, 17^3 template at +-9, so the search
          takes the reference's FP32 FFT branch; tricubic, three ADMM steps;
  bspline 56 x 64 x 72 float32 beads, B-spline interpolation, a featureless block (flat subsets fail the
          precompute and the initial guess), the default ADMM early stop.
"""

from __future__ import annotations

import hashlib

import numpy as np

from pyaldvc_b200 import synthetic as syn

F_AFFINE = np.array([[0.01, 0.004, 0.0], [0.002, -0.008, 0.003], [0.0, -0.002, 0.012]])

PASS_CASES = {
    "affine": dict(shape=(56, 64, 72), seed=61, t=(1.3, -0.7, 0.4), sigma=1.5, uint16=False, mask=False, flat=False,
                   para=dict(winsize=(16, 16, 16), winstepsize=(8, 8, 8), search_radius=(4, 4, 4), interp_method="cubic",
                             admm_max_iter=3)),
    "masked": dict(shape=(56, 64, 72), seed=61, t=(1.3, -0.7, 0.4), sigma=1.5, uint16=False, mask=True, flat=False,
                   para=dict(winsize=(16, 16, 16), winstepsize=(8, 8, 8), search_radius=(4, 4, 4), interp_method="linear",
                             admm_max_iter=3, admm_tol=1e-9)),
    "fft": dict(shape=(80, 80, 88), seed=62, t=(3.4, -2.2, 4.6), sigma=2.0, uint16=True, poisson=1000.0, mask=False, flat=False,
                para=dict(winsize=(32, 32, 32), winstepsize=(12, 12, 12), search_radius=(9, 9, 9), interp_method="cubic",
                          admm_max_iter=3, admm_tol=1e-9)),
    "bspline": dict(shape=(56, 64, 72), seed=63, t=(-0.6, 1.1, 0.8), sigma=1.5, uint16=False, mask=False, flat=True,
                    para=dict(winsize=(16, 16, 16), winstepsize=(8, 8, 8), search_radius=(4, 4, 4), interp_method="bspline",
                              admm_max_iter=4)),
}
# parameters every pass case shares (the reference's names); beta fixed, FEM global step, PCG solver
PASS_COMMON = dict(init_guess_method="ncc", global_shift=False, beta=1e-3, mu=1e-3, subpb2_method="fem", global_solver="pcg",
                   gradient_mode="stored", subset_split=False)


def sha(a) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def pass_pair(name):
    """(f, g, mask or None, displacement function) of a pass case, raw (before normalisation)."""
    c = PASS_CASES[name]
    shape = c["shape"]
    centre = tuple((s - 1) / 2 for s in shape[::-1])
    disp = syn.affine(F_AFFINE, c["t"], centre)
    pair = syn.bead_pair(shape, density=0.02, sigma=c["sigma"], seed=c["seed"], disp=disp, noise=0.01,
                         poisson_photons=c.get("poisson"), uint16_max=4095 if c["uint16"] else None)
    f, g = pair.f, pair.g
    if c["flat"]:  # a featureless block in both frames
        f = f.copy()
        g = g.copy()
        f[4:24, 4:26, 4:28] = f.dtype.type(0.2)
        g[4:24, 4:26, 4:28] = g.dtype.type(0.2)
    mask = None
    if c["mask"]:
        nz, ny, nx = shape
        z, y, x = np.ogrid[:nz, :ny, :nx]
        mask = ((x - 30.0) ** 2 + (y - 34.0) ** 2 + (z - 26.0) ** 2) <= 27.0**2
    return f, g, mask, disp


NCC_SHAPE = (108, 116, 124)
NCC_T = (19.3, -17.6, 6.2)
NCC_F = np.array([[0.006, 0.0, 0.002], [0.0, -0.004, 0.0], [0.003, 0.0, 0.008]])
NCC_SEARCHES = {
    "r9": dict(subset=(16, 16, 16), radius=(9, 9, 9), shift=True),
    "r16": dict(subset=(16, 16, 16), radius=(16, 16, 16), shift=True),
    "aniso": dict(subset=(16, 12, 20), radius=(12, 10, 14), shift=True),
}
NCC_EXPAND = dict(subset=(16, 16, 16), radius=(8, 8, 8))  # +-8 direct, then +-16 and +-32 on the FFT branch


def ncc_pair():
    """Raw bead pair of the FFT-branch searches: a large translation plus a small affine part."""
    centre = tuple((s - 1) / 2 for s in NCC_SHAPE[::-1])
    return syn.bead_pair(NCC_SHAPE, density=0.02, sigma=1.5, seed=64, disp=syn.affine(NCC_F, NCC_T, centre), noise=0.01)


def ncc_coords():
    """Node centres [x, y, z] every 13 voxels, 20 voxels or more from the faces."""
    axes = [np.arange(20, n - 20, 13) for n in NCC_SHAPE]
    zz, yy, xx = np.meshgrid(*axes, indexing="ij")
    return np.stack([xx.ravel(), yy.ravel(), zz.ravel()], 1).astype(np.int64)


def ncc_shift(coords):
    """The integer prior shift of the searches that have one: the rounded field at the nodes, off by up to
    two voxels so the peaks are not all at the window centre."""
    centre = tuple((s - 1) / 2 for s in NCC_SHAPE[::-1])
    u = np.column_stack(syn.affine(NCC_F, NCC_T, centre)(*(coords[:, k].astype(float) for k in range(3))))
    off = np.stack([(np.arange(len(coords)) * 7 + k) % 5 - 2 for k in range(3)], 1)
    return np.round(u).astype(np.int64) + off


# Frame series of golden_series.npz (the reference's run_aldvc over three frames): frame 0 and two frames of the same
# beads moved by growing affine fields, each frame with its own noise; ws 16 / step 8, direct NCC +-4, tricubic, three
# ADMM steps at most with the reference's early stop.  Cases: accumulative with the "previous" initial guess (frame
# 2 starts from frame 1's field), incremental with the cubic and the linear cumulative composition.
SERIES_SHAPE = (56, 64, 72)
SERIES_CASES = {
    "accum_prev": dict(reference_mode="accumulative", init_guess_method="previous", cumulative_interp="cubic"),
    "incr_cubic": dict(reference_mode="incremental", init_guess_method="ncc", cumulative_interp="cubic"),
    "incr_linear": dict(reference_mode="incremental", init_guess_method="ncc", cumulative_interp="linear"),
}
SERIES_PARA = dict(winsize=(16, 16, 16), winstepsize=(8, 8, 8), search_radius=(4, 4, 4), interp_method="cubic", admm_max_iter=3)


def series_frames():
    """Three float32 frames: the beads of frame 0 moved by affine fields with translations (0.9, -0.5, 0.3) and
    (2.1, -1.3, 0.8) and gradients F_AFFINE, 2 F_AFFINE about the volume centre."""
    shape = SERIES_SHAPE
    centre = tuple((s - 1) / 2 for s in shape[::-1])
    centres, peaks = syn.draw_beads(shape, 0.02, 81)
    out = []
    for k, (t, scale) in enumerate((((0.0, 0.0, 0.0), 0.0), ((0.9, -0.5, 0.3), 1.0), ((2.1, -1.3, 0.8), 2.0))):
        disp = syn.affine(scale * F_AFFINE, t, centre)
        vol = syn.render_beads(shape, syn.displace_beads(centres, disp), peaks, 1.5).astype(np.float64)
        vol = vol + np.random.default_rng(90 + k).normal(0.0, 0.01, size=vol.shape)
        out.append(vol.astype(np.float32))
    return out
