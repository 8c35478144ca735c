"""CPU: the oracle's separable volume filters against the reference's own outputs (tests/golden/
golden_volume_ops.npz, made by tests/golden/make_golden.py from io/volume_ops.py:200-222).

The Gaussian presmoothing is bit-identical.  The B-spline prefilter is bit-identical on lines of 7 or more
samples; on shorter mirrored lines the exact result of the filter is a short combination of float32 inputs that
often lies on a float32 rounding tie, where the oracle's FP64 sum and scipy's recursion can round to neighbours,
so those lines are held to one float32 step of the largest coefficient.
"""

from __future__ import annotations

import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope="module")
def vg():
    with np.load(os.path.join(HERE, "golden", "golden_volume_ops.npz")) as z:
        return {k: z[k] for k in z.files}


def test_oracle_gaussian_presmooth_matches_reference(oracle_mod, vg):
    for s in ("0.8", "2.0"):
        np.testing.assert_array_equal(oracle_mod.presmooth_volume(vg["vol"], float(s)), vg[f"gauss_{s}"])
    np.testing.assert_array_equal(oracle_mod.presmooth_volume(vg["small"], 1.0), vg["small_gauss_1.0"])
    np.testing.assert_array_equal(oracle_mod.presmooth_volume(vg["vol"], 0.0), vg["vol"])


def test_oracle_bspline_prefilter_matches_reference(oracle_mod, vg):
    np.testing.assert_array_equal(oracle_mod.prefilter_bspline(vg["vol"]), vg["bspline"])
    got, ref = oracle_mod.prefilter_bspline(vg["small"]), vg["small_bspline"]
    np.testing.assert_allclose(got, ref, rtol=0, atol=2.0**-22 * np.abs(ref).max())


def test_oracle_bspline_coefficients_interpolate_the_volume(oracle_mod, vg):
    """Sampling the coefficients with the cubic B-spline at the voxel centres gives back the volume."""
    c = oracle_mod.prefilter_bspline(vg["vol"]).astype(np.float64)
    b = np.array([1.0, 4.0, 1.0]) / 6.0
    inner = c
    for ax in range(3):
        inner = b[0] * np.roll(inner, 1, ax) + b[1] * inner + b[2] * np.roll(inner, -1, ax)
    v = vg["vol"].astype(np.float64)
    sl = (slice(1, -1),) * 3
    assert np.abs(inner[sl] - v[sl]).max() < 1e-5 * np.abs(v).max()
