"""CPU: the inputs and the oracle of the initial-guess pipeline against the reference's own outputs
(tests/golden/golden_init_guess.npz, made by tests/golden/make_golden.py from solver/integer_search.py:235-694
and utils/).

The fixture stores no volumes: the tests rebuild the seeded bead pairs with pyaldvc_b200.synthetic and check their
SHA-256 against the reference-normalised volumes the fixture was made from.
"""

from __future__ import annotations

import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))

import init_guess_inputs as IG  # noqa: E402


@pytest.fixture(scope="module")
def ig():
    with np.load(os.path.join(HERE, "golden", "golden_init_guess.npz")) as z:
        return {k: z[k] for k in z.files}


def test_regenerated_inputs_are_the_reference_inputs(ig):
    pf, pg = IG.normalised(IG.raw_pc_pair())
    assert IG.sha(pf) == str(ig["pc_sha_f"]) and IG.sha(pg) == str(ig["pc_sha_g"])
    yf, yg = IG.normalised(IG.raw_py_pair())
    assert IG.sha(yf) == str(ig["py_sha_f"]) and IG.sha(yg) == str(ig["py_sha_g"])


def test_oracle_block_downsample_matches_reference(oracle_mod, ig):
    v = ig["bd_vol"]
    for fac in (2, 3, 4):
        ref = ig[f"bd_{fac}"]
        got = oracle_mod.block_downsample(v, fac)
        assert got.shape == ref.shape
        # the reference sums the fac^3 voxels in float32 (numpy's order), the oracle in FP64: they differ by at most
        # the float32 sum's rounding, fac^3 half-steps of the largest magnitude, over fac^3
        np.testing.assert_allclose(got, ref, rtol=0, atol=2.0**-24 * np.abs(v).max())


def test_oracle_phase_correlation_matches_reference(oracle_mod, ig):
    pf, pg = IG.normalised(IG.raw_pc_pair())
    np.testing.assert_array_equal(oracle_mod.phase_correlation_shift(pf, pg), ig["pc_shift"])
    np.testing.assert_array_equal(oracle_mod.phase_correlation_shift(pf, pg, 24), ig["pc_shift_md24"])
