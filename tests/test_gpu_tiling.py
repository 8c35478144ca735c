"""GPU: the tiled pass (tiling.run_pass_tiled, volumes in host memory, every step box by box) against the pass on
whole device volumes (pipeline.run_pass).

The reference's own bar for its tiling (tests/test_tiling.py:98-170): identical statuses, iteration counts and
rejected nodes, displacements within 1e-9 voxel (a box-local x0 rounds ``x0 + P[9]`` differently; the lean
kernels here form sample positions relative to the node centre, so they usually agree exactly).  Cases:

- the four golden pass pairs (cubic with early stop, masked trilinear, B-spline with a flat block, and the uint16
  pair whose 17^3 template takes the FFT engine), boxes of 64 voxels (16 or more per pass, the integer search in
  its own boxes);
- the default initial guess (global phase-correlation shift and the coarse-to-fine pyramid) on a pair larger than
  128 voxels per axis, so the shift and the coarse levels use block means built slab by slab;
- statistics accumulated over several slabs (normalisation within FP64 rounding of the one-slab value);
- a small device cache, so every stage streams its boxes again;
- the Gaussian presmoothing, run on boxes grown by its reach.
"""

from __future__ import annotations

import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))

import pass_inputs as PI  # noqa: E402

pytestmark = pytest.mark.gpu

U_TOL = 1e-9  # voxel
F_TOL = 1e-11


def _np(t):
    return t.detach().cpu().numpy()


def _params(name, **over):
    from pyaldvc_b200.pipeline import PassParams

    c = PI.PASS_CASES[name]["para"]
    p = PassParams(winsize=c["winsize"], winstepsize=c["winstepsize"], search_radius=c["search_radius"],
                   interp_method=c["interp_method"], admm_max_iter=c["admm_max_iter"], admm_tol=c.get("admm_tol", 1e-2),
                   init_guess_method="ncc", global_shift=False, beta=PI.PASS_COMMON["beta"], mu=PI.PASS_COMMON["mu"], autotune=False,
                   threads=128, tile_disp_margin=2)
    for k, v in over.items():
        setattr(p, k, v)
    return p


def _whole(f, g, p, mask=None):
    import torch

    from pyaldvc_b200.pipeline import run_pass

    cu = lambda a: None if a is None else torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    return run_pass(cu(f), cu(g), p, cu(None if mask is None else mask.astype(np.uint8)))


def _same(a, b, what, tol=0.0):
    a, b = _np(a), _np(b)
    assert a.shape == b.shape, what
    assert np.array_equal(np.isnan(a), np.isnan(b)) if a.dtype.kind == "f" else True, f"{what}: NaN pattern"
    if tol == 0.0:
        ok = (a == b) | (np.isnan(a) & np.isnan(b)) if a.dtype.kind == "f" else a == b
        assert ok.all(), f"{what}: differs at {np.flatnonzero(~ok.reshape(-1))[:8]}"
    else:
        d = np.nanmax(np.abs(a - b)) if a.size else 0.0
        assert d <= tol, f"{what}: max |diff| {d:.3e} > {tol:g}"


def _compare(t, w, what, u_tol=U_TOL, f_tol=F_TOL):
    _same(t.valid, w.valid, f"{what} valid")
    _same(t.coords, w.coords, f"{what} coords")
    _same(t.U0, w.U0, f"{what} U0", u_tol)
    for k in ("status_local", "n_iter_local", "status", "n_iter"):
        _same(getattr(t, k), getattr(w, k), f"{what} {k}")
    assert t.admm_steps == w.admm_steps, what
    for k, tol in (("U_local", u_tol), ("F_local", f_tol), ("U", u_tol), ("F", f_tol), ("zncc", 1e-12)):
        _same(getattr(t, k), getattr(w, k), f"{what} {k}", tol)


@pytest.mark.parametrize("name", list(PI.PASS_CASES))
def test_tiled_pass_matches_whole_volume_pass(name):
    from pyaldvc_b200.tiling import run_pass_tiled

    f, g, mask, _ = PI.pass_pair(name)
    edge = 112 if name == "fft" else 64
    p = _params(name, tile_strain_margin=0.0 if name == "fft" else 0.25)
    w = _whole(f, g, p, mask)
    t = run_pass_tiled(f, g, p, mask=mask, edge=edge)
    _compare(t, w, name)
    rec = t.tiles.stages
    assert rec["icgn12"]["boxes"] > 1, rec
    if name != "fft":  # the FFT case's 33^3 subsets and 17^3 templates at +-9: one precompute and one search box
        assert rec["precompute"]["boxes"] > 1 and rec["ncc"]["boxes"] > 1, rec
    assert rec["icgn12"]["max_voxels"] < np.prod(f.shape)
    if p.use_global_step and t.admm_steps > 1:
        assert rec["icgn3"]["calls"] == t.admm_steps - 1


def _large_pair():
    """96 x 144 x 160 float32 beads with a 5-voxel translation plus the affine field: more than 128 voxels along x,
    so the global shift block-averages by 2, and room for one coarse pyramid level."""
    from pyaldvc_b200 import synthetic as syn

    shape = (96, 144, 160)
    centre = tuple((s - 1) / 2 for s in shape[::-1])
    disp = syn.affine(PI.F_AFFINE, (5.3, -4.6, 2.4), centre)
    pair = syn.bead_pair(shape, density=0.02, sigma=1.5, seed=71, disp=disp, noise=0.01)
    return pair.f, pair.g


def test_tiled_default_initial_guess_streams_block_means():
    from pyaldvc_b200.tiling import run_pass_tiled

    f, g = _large_pair()
    p = _params("affine", winsize=(20, 20, 20), winstepsize=(12, 12, 12), search_radius=(6, 6, 6), init_guess_method="pyramid",
                global_shift=True, admm_max_iter=2)
    w = _whole(f, g, p)
    slab = 20 * 144 * 160  # slabs of 20 planes: the block means cross slab boundaries only between whole blocks
    t = run_pass_tiled(f, g, p, edge=80, slab_voxels=slab)
    assert w.init_info["method"] == "pyramid" and t.init_info["levels"] == w.init_info["levels"]
    np.testing.assert_array_equal(t.init_info["global_shift"], w.init_info["global_shift"])
    assert w.init_info["global_shift"] is not None and np.abs(w.init_info["global_shift"]).max() > 0
    # several slabs accumulate the normalisation moments in another grouping: FP64 rounding of the statistics
    # can move a normalised voxel by one float32 step, so the field agrees to far below the solver's tolerance
    _same(t.valid, w.valid, "valid")
    _same(t.status, w.status, "status")
    _same(t.U, w.U, "U", 1e-6)
    assert t.frames.boxes_loaded > 10


def test_tiled_pass_one_slab_normalisation_is_exact_and_uint16():
    """One slab: the moments are aldvc_normalize's own, so the uint16 pair normalises bit for bit."""
    import torch

    from pyaldvc_b200 import kernels as K
    from pyaldvc_b200.tiling import Box, HostFrames

    f, g, _, _ = PI.pass_pair("fft")
    p = _params("fft")
    fr = HostFrames(f, g, p)
    whole = K.normalize(torch.from_numpy(f).cuda())
    box = Box((10, 20, 30), (40, 30, 50))
    got = fr._frame("f", box)
    assert torch.equal(got, whole[box.slices])
    fr_multi = HostFrames(f, g, p, slab_voxels=13 * 80 * 88)
    assert len(fr_multi.slabs()) > 3
    d = (fr_multi._frame("f", box) - got).abs().max().item()
    assert d <= 2e-6


def test_tiled_pass_with_presmoothing_and_no_cache():
    from pyaldvc_b200.tiling import run_pass_tiled

    f, g, mask, _ = PI.pass_pair("affine")
    p = _params("affine", prefilter_sigma=1.0)
    w = _whole(f, g, p)
    t = run_pass_tiled(f, g, p, edge=72, cache_bytes=0)
    _compare(t, w, "presmoothed")
    assert t.frames.cache_hits == 0


def test_bspline_box_coefficients_equal_the_whole_volume_prefilter():
    import torch

    from pyaldvc_b200 import kernels as K
    from pyaldvc_b200.tiling import Box, HostFrames

    f, g, _, _ = PI.pass_pair("bspline")
    p = _params("bspline")
    fr = HostFrames(f, g, p)
    whole = K.bspline_prefilter(K.normalize(torch.from_numpy(g).cuda()))
    for box in (Box((0, 5, 9), (30, 40, 50), (False, True, True, True, True, True)), Box((20, 30, 40), (36, 34, 32))):
        v = fr.local_volumes(box, quads=True)
        assert torch.equal(v["g"], whole[box.slices])
        assert torch.equal(v["g4"], K.make_quads(v["g"]))


def test_tiled_pass_with_uneven_subsets_and_masks():
    """Per-node subset shapes (the precompute's per-node form in every box), a reference mask and a deformed-frame
    mask (NaN in the interpolant, 0 in the search input, each cut per box): the tiled pass equals the whole one."""
    import torch

    from pyaldvc_b200.pipeline import run_pass
    from pyaldvc_b200.tiling import run_pass_tiled

    f, g, mask, _ = PI.pass_pair("masked")
    nz, ny, nx = f.shape
    z, y, x = np.ogrid[:nz, :ny, :nx]
    g_mask = ~((x - 50.0) ** 2 + (y - 20.0) ** 2 + (z - 40.0) ** 2 <= 6.0**2)  # a hole in the deformed frame

    def winsize(c):  # 12 to 16 voxels per axis with the node's x position
        c = np.asarray(c)
        w = 12 + 2 * ((c[:, 0] // 16) % 3)
        return np.stack([w, np.full_like(w, 16), np.full_like(w, 14)], 1)

    p = _params("masked", node_winsize=winsize, interp_method="cubic")
    cu = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    w = run_pass(cu(f), cu(g), p, cu(mask.astype(np.uint8)), g_mask=cu(g_mask.astype(np.uint8)))
    t = run_pass_tiled(f, g, p, mask=mask, g_mask=g_mask, edge=64)
    _compare(t, w, "uneven masked")
    assert t.precompute_form == "per_node" and t.tiles.stages["icgn12"]["boxes"] > 1
