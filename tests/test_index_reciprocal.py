"""The NCC kernels split a linear index r into (row, column) as int(((float)r + 0.5f) * (1.0f / (float)d)) instead of an
integer division by a runtime extent d (`sweep_lin` and `fdivi` in pyaldvc_b200/csrc/ncc.cu).  The split is exact for
0 <= r < 2^22: the true quotient (r + 0.5) / d lies at least 0.5 / d from an integer, while the reciprocal's and the
product's roundings move it by less than that.  This checks the claim in IEEE float32 arithmetic (numpy rounds each
float32 operation to nearest, as the device's division and multiply do) at every place it could fail: both sides of
every multiple of d below 2^22, for every extent the kernels pass (map rows and columns up to 2 * 256 + 1, template and
neighbour-box sides up to 1026, padded template rows)."""

from __future__ import annotations

import numpy as np

LIMIT = 1 << 22


def _split(r: np.ndarray, d: int) -> np.ndarray:
    inv = np.float32(1.0) / np.float32(d)
    return ((r.astype(np.float32) + np.float32(0.5)) * inv).astype(np.int64)


def test_reciprocal_split_is_exact_below_2_pow_22():
    for d in range(1, 1100):
        k = np.arange(0, LIMIT // d + 1, dtype=np.int64) * d
        r = np.concatenate([k - 1, k, k + 1])
        r = r[(r >= 0) & (r < LIMIT)]
        np.testing.assert_array_equal(_split(r, d), r // d, err_msg=f"divisor {d}")


def test_reciprocal_split_every_index_of_small_tiles():
    for d in (3, 17, 19, 20, 25, 27, 33, 35, 49, 65):
        r = np.arange(0, 70 * 70 * 70, dtype=np.int64)
        np.testing.assert_array_equal(_split(r, d), r // d, err_msg=f"divisor {d}")
