"""GPU: the initial-guess pipeline around the NCC kernel against the reference's own outputs
(tests/golden/golden_init_guess.npz: solver/integer_search.py:235-694, utils/outlier_detection.py:135,
utils/inpaint.py:35) and the oracle.

Parity bar: integer results (phase-correlation shifts, pyramid levels, per-level radii, subsets and peak counts,
expansions, ok flags, median-test flags) identical; the pyramid's sub-voxel displacements within 1e-6 voxel and its
peak values within 1e-9 (FP64 re-scores on both sides; the inpainting between levels is a CG solve to 1e-12 here
and a direct solve in the reference); PCE within 1e-5 relative (map energy from the FP32 map); block means within
one float32 step of the reference's float32 sums.
"""

from __future__ import annotations

import os
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))

import init_guess_inputs as IG  # noqa: E402


@pytest.fixture(scope="module")
def ig():
    with np.load(os.path.join(HERE, "golden", "golden_init_guess.npz")) as z:
        return {k: z[k] for k in z.files}


def _dev(a):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def test_block_downsample(oracle_mod, ig):
    from pyaldvc_b200 import integer_search as IS

    v = ig["bd_vol"]
    for fac in (2, 3, 4):
        got = IS.block_downsample(v, fac)
        np.testing.assert_allclose(got, ig[f"bd_{fac}"], rtol=0, atol=2.0**-24 * np.abs(v).max())
        np.testing.assert_allclose(got, oracle_mod.block_downsample(v, fac), rtol=0, atol=2.0**-24 * np.abs(v).max())
    np.testing.assert_array_equal(IS.block_downsample(v, 1), v)


def test_volume_stats_and_voi_normalisation():
    """voi_mean_std / normalize_volume over a VOI box (io/volume_ops.py:74-121), against their FP64 formula."""
    import torch

    from pyaldvc_b200 import kernels as K

    rng = np.random.default_rng(4)
    raw = rng.integers(0, 4096, (30, 41, 52)).astype(np.uint16)
    box = (3, 27, 5, 40, 0, 33)
    z0, z1, y0, y1, x0, x1 = box
    sub = raw[z0:z1, y0:y1, x0:x1].astype(np.float64)
    pilot = float(raw[(z0 + z1) // 2, (y0 + y1) // 2, (x0 + x1) // 2])
    d = sub - pilot
    ms = d.sum() / d.size
    sd = np.sqrt(max((d * d).sum() / d.size - ms * ms, 0.0))
    mean = pilot + ms
    for vol in (_dev(raw), _dev(raw.astype(np.float32))):
        st = K.volume_stats(vol, box).cpu().numpy()
        np.testing.assert_allclose(st, [mean, sd], rtol=1e-13)
        out, _ = K.normalize_voi(vol, box)
        ref = ((raw.astype(np.float64) - mean) * (1.0 / sd)).astype(np.float32)
        got = out.cpu().numpy()
        np.testing.assert_allclose(got, ref, rtol=0, atol=np.spacing(np.abs(ref).max()))
        assert np.mean(got == ref) > 0.999
    flat = torch.full((4, 5, 6), 7.0, device="cuda")
    out, st = K.normalize_voi(flat, None)
    assert float(st[1]) == 0.0 and float(out.abs().max()) == 0.0  # std < 1e-12 is taken as 1


def test_phase_correlation_shift_matches_reference(ig):
    from pyaldvc_b200 import integer_search as IS

    pf, pg = IG.normalised(IG.raw_pc_pair())
    np.testing.assert_array_equal(IS.phase_correlation_shift(pf, pg), ig["pc_shift"])
    np.testing.assert_array_equal(IS.phase_correlation_shift(pf, pg, None, 24), ig["pc_shift_md24"])
    # the known translation (6.3, -9.6, 4.2) to within the peak's voxel
    assert np.abs(IS.phase_correlation_shift(pf, pg) - np.array(IG.PC_T)).max() < 1.0


def test_median_test_and_inpainting_match_reference(ig):
    import torch

    from pyaldvc_b200 import kernels as K

    field, valid = ig["mt_field"], ig["mt_valid"]
    gs = field.shape[:3]
    f = torch.from_numpy(np.where(valid[..., None], field, np.nan).reshape(-1, 3)).cuda().contiguous()
    flag, _ = K.median_test(f, gs, _dev(valid.reshape(-1).astype(np.uint8)), 2.0)
    np.testing.assert_array_equal(flag.cpu().numpy().reshape(gs).astype(bool), ig["mt_flag"])
    holes = ig["fill_in"]
    unk = np.isnan(holes)
    v = torch.from_numpy(np.where(unk, 0.0, holes).reshape(-1, 1)).cuda().contiguous()
    K.inpaint(v, gs, _dev(unk.reshape(-1).astype(np.uint8)))
    np.testing.assert_allclose(v.cpu().numpy().reshape(gs), ig["fill_out"], rtol=0, atol=1e-8)


def test_pyramid_search_matches_reference(ig):
    from pyaldvc_b200 import integer_search as IS

    yf, yg = IG.normalised(IG.raw_py_pair())
    assert IS.auto_pyramid_levels(IG.PY_SHAPE, IG.PY_SUBSET, IG.PY_RADIUS, f=yf) == int(ig["py_levels"])
    shift = IS.phase_correlation_shift(yf, yg)
    np.testing.assert_array_equal(shift, ig["py_shift"])
    info = IS.pyramid_search(yf, yg, ig["py_coords"], tuple(ig["py_grid"]), IG.PY_SUBSET, IG.PY_RADIUS, 0, global_shift=shift)
    assert info["levels"] == int(ig["py_levels"])
    assert info["expansions"] == int(ig["py_expansions"])
    np.testing.assert_array_equal([d["n_ok"] for d in info["per_level"]], ig["py_level_nok"])
    np.testing.assert_array_equal([d["radius"] for d in info["per_level"]], ig["py_level_radius"])
    np.testing.assert_array_equal([d["subset"] for d in info["per_level"]], ig["py_level_subset"])
    np.testing.assert_array_equal(info["ok"], ig["py_ok"])
    np.testing.assert_array_equal(info["clipped"], ig["py_clipped"])
    np.testing.assert_allclose(info["disp"], ig["py_disp"], rtol=0, atol=1e-6)
    ok = ig["py_ok"]
    np.testing.assert_allclose(info["cc"][ok], ig["py_cc"][ok], rtol=0, atol=1e-9)
    # PCE divides by the energy of the whole map, summed over the FP32 map here and the FP64 map in the reference
    np.testing.assert_allclose(info["pce"][ok], ig["py_pce"][ok], rtol=1e-5)


def test_pass_initial_guess_methods():
    """Full passes on the 96^3 affine pair (translation (5.4, -7.2, 9.7) plus shear) seeded by the pyramid search
    and by one full-resolution NCC search, both with the global pre-shift: every node that converges from both
    seeds reaches the same solution (within IC-GN's stopping tolerance), within 0.02 voxel RMS of the truth.  Nodes within about 10 voxels of a face
    leave the volume under the translation (status 2) whatever the seed.  A zero seed runs to completion."""
    import torch

    from pyaldvc_b200.pipeline import PassParams, run_pass

    pair = IG.raw_py_pair()
    f, g = (torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in (pair.f, pair.g))
    out = {}
    for method in ("pyramid", "ncc", "zero"):
        p = PassParams(winsize=(20, 20, 20), winstepsize=(10, 10, 10), search_radius=(12, 12, 12), init_guess_method=method,
                       global_shift=method != "zero", use_global_step=False, autotune=False)
        res = run_pass(f, g, p)
        assert res.init_info["method"] == method
        out[method] = res
    assert out["pyramid"].init_info["levels"] >= 1
    coords = out["ncc"].coords.cpu().numpy().astype(float)
    truth = np.column_stack(pair.disp(*coords.T))
    ok = (out["pyramid"].status.cpu().numpy() == 0) & (out["ncc"].status.cpu().numpy() == 0)
    assert ok.mean() > 0.6
    Up, Un = (out[m].U.cpu().numpy() for m in ("pyramid", "ncc"))
    # IC-GN stops once its update falls below dp_tol = 1e-3: runs from two seeds end within a few such steps
    np.testing.assert_allclose(Up[ok], Un[ok], rtol=0, atol=5e-3)
    assert np.mean(np.abs(Up[ok] - Un[ok]) < 1e-3) > 0.99
    assert np.sqrt(np.mean((Up[ok] - truth[ok]) ** 2)) < 0.02
    assert np.isfinite(out["zero"].U.cpu().numpy()).all()
