"""GPU: the integer search against the reference's FFT branch (tests/golden/golden_ncc_fft.npz).

Above 3e7 offset x template-voxel products per node the reference's CPU search correlates with FP32 FFTs
(integer_search.py:395, :418-443) and takes the first maximum of that FP32 map.  Every engine here scores its
FP32 map's near-maximal offsets again in FP64 (the exact map of the direct formula) and takes the first maximum
of those.  The two rules pick the same integer peak unless the exact map's two best offsets lie within the FFT
map's rounding of each other: the tests below require identical ok / clipped flags and integer peaks at every
node whose exact top-two gap exceeds 1e-5, count the near-tie nodes, and require the engines' own choice there
to be the exact map's first maximum.  Sub-voxel displacements and peak values differ from the reference's only
by the FFT map's rounding (disp 1e-4 voxel, cc 2e-6).
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

ENGINES = {"tiled": 0, "plain": 1, "fft": 2, "fft_stockham": 3, "fft_cluster": 4}
NEAR_TIE = 1e-5


@pytest.fixture(scope="module")
def gn():
    with np.load(os.path.join(HERE, "golden", "golden_ncc_fft.npz")) as z:
        return {k: z[k] for k in z.files}


@pytest.fixture(scope="module")
def ncc_in(oracle_mod, gn):
    pair = PI.ncc_pair()
    f, g = oracle_mod.normalize_volume(pair.f), oracle_mod.normalize_volume(pair.g)
    assert PI.sha(f) == str(gn["sha_f"]) and PI.sha(g) == str(gn["sha_g"])
    return f, g, gn["coords"], gn["shift"]


def _exact_top2(oracle_mod, f, g, coords, subset, radius, shift):
    """First maximum (flat index) and the gap to the second-best offset of the exact FP64 map, per node."""
    hx, hy, hz = (int(w) // 2 for w in subset)
    rx, ry, rz = radius
    nz, ny, nx = f.shape
    wx, wy, wz = 2 * hx + 1 + 2 * rx, 2 * hy + 1 + 2 * ry, 2 * hz + 1 + 2 * rz
    sh = np.zeros_like(coords) if shift is None else shift
    wx0 = np.clip(coords[:, 0] + sh[:, 0] - hx - rx, 0, nx - wx)
    wy0 = np.clip(coords[:, 1] + sh[:, 1] - hy - ry, 0, ny - wy)
    wz0 = np.clip(coords[:, 2] + sh[:, 2] - hz - rz, 0, nz - wz)
    maps = np.empty((len(coords), 2 * rz + 1, 2 * ry + 1, 2 * rx + 1))
    oracle_mod.zncc_direct(f, g, coords, hx, hy, hz, rx, ry, rz, wx0, wy0, wz0, np.ones(len(coords), bool), maps)
    flat = maps.reshape(len(coords), -1)
    top = np.sort(flat, axis=1)[:, -2:]
    return np.argmax(flat, axis=1), top[:, 1] - top[:, 0], (wx0, wy0, wz0)


def _compare(oracle_mod, f, g, coords, shift, subset, radius, res, ref, what):
    ok = ref["ok"]
    np.testing.assert_array_equal(res["ok"], ok, err_msg=f"{what}: ok")
    d = np.abs(res["disp"] - ref["disp"])
    moved = np.flatnonzero(ok & (np.nanmax(d, axis=1) > 0.5))  # a different integer peak
    same = ok.copy()
    same[moved] = False
    np.testing.assert_array_equal(res["clipped"][same], ref["clipped"][same], err_msg=f"{what}: clipped")
    np.testing.assert_allclose(res["disp"][same], ref["disp"][same], rtol=0, atol=1e-4, err_msg=f"{what}: disp")
    np.testing.assert_allclose(res["cc"][same], ref["cc"][same], rtol=0, atol=2e-6, err_msg=f"{what}: cc")
    np.testing.assert_allclose(res["pce"][same], ref["pce"][same], rtol=2e-3, err_msg=f"{what}: pce")
    if moved.size:
        # the engines' peak there must be the exact map's first maximum, and the reference's a near tie of it
        sel = moved
        arg, gap, (wx0, wy0, wz0) = _exact_top2(oracle_mod, f, g, coords[sel], subset, radius,
                                                None if shift is None else shift[sel])
        assert np.all(gap < NEAR_TIE), f"{what}: peaks differ at nodes {sel} whose exact top-two gap is {gap}"
        hx, hy, hz = (int(w) // 2 for w in subset)
        vz, vy, vx = (2 * r + 1 for r in radius[::-1])
        pz, py, px = np.unravel_index(arg, (vz, vy, vx))
        exact = np.column_stack([wx0 + px + hx - coords[sel, 0], wy0 + py + hy - coords[sel, 1], wz0 + pz + hz - coords[sel, 2]])
        np.testing.assert_array_less(np.abs(res["disp"][sel] - exact), 1.0, err_msg=f"{what}: engine peak is not the exact one")
    return moved.size


@pytest.mark.parametrize("engine", list(ENGINES))
@pytest.mark.parametrize("name", list(PI.NCC_SEARCHES))
def test_ncc_search_matches_reference_fft_branch(oracle_mod, gn, ncc_in, name, engine):
    from pyaldvc_b200.integer_search import ncc_search

    f, g, coords, shift = ncc_in
    c = PI.NCC_SEARCHES[name]
    sh = shift if c["shift"] else None
    res = ncc_search(f, g, coords, c["subset"], c["radius"], sh, engine=ENGINES[engine])
    ref = {k: gn[f"{name}_{k}"] for k in ("disp", "cc", "pce", "clipped", "ok")}
    n_ties = _compare(oracle_mod, f, g, coords, sh, c["subset"], c["radius"], res, ref, f"{name}/{engine}")
    assert n_ties <= 0.02 * len(coords), f"{name}/{engine}: {n_ties} near-tie nodes"


@pytest.mark.parametrize("engine", ["tiled", "fft"])
def test_ncc_expansion_matches_reference_fft_branch(oracle_mod, gn, ncc_in, engine):
    """+-8 (the reference's direct branch), then +-16 and +-32 (its FFT branch) on the clipped nodes."""
    from pyaldvc_b200.integer_search import ncc_search_expanding

    f, g, coords, _ = ncc_in
    res = ncc_search_expanding(f, g, coords, PI.NCC_EXPAND["subset"], PI.NCC_EXPAND["radius"], engine=ENGINES[engine])
    assert res["expansions"] == int(gn["expand_expansions"]) == 2
    assert tuple(res["radius"]) == tuple(int(r) for r in gn["expand_radius"])
    ref = {k: gn[f"expand_{k}"] for k in ("disp", "cc", "pce", "clipped", "ok")}
    n_ties = _compare(oracle_mod, f, g, coords, None, PI.NCC_EXPAND["subset"], tuple(res["radius"]), res, ref, f"expand/{engine}")
    assert n_ties <= 0.02 * len(coords)


@pytest.mark.parametrize("name", ["r16", "r9", "t15r16"])
def test_cluster_engine_equals_three_pass_engine(gn, ncc_in, name):
    """The cluster form runs every line through the same transforms in the same order as the three passes of the
    in-register engine: identical integer peaks, sub-voxel displacements and peak values.  The PCE energy sums the
    map in other blocks (a cluster CTA's planes instead of a pass-3 CTA's), so it agrees to FP64 rounding.  At +-9
    the 36-point box takes the three passes in both (its row pairs do not fit one cluster)."""
    from pyaldvc_b200.integer_search import ncc_search

    f, g, coords, shift = ncc_in
    # t15r16: a 15^3 template at +-16, a 47-voxel window in a 48-point box (the cluster form's other length)
    c = PI.NCC_SEARCHES[name] if name in PI.NCC_SEARCHES else dict(subset=(14, 14, 14), radius=(16, 16, 16))
    a = ncc_search(f, g, coords, c["subset"], c["radius"], shift, engine=ENGINES["fft"])
    b = ncc_search(f, g, coords, c["subset"], c["radius"], shift, engine=ENGINES["fft_cluster"])
    for k in ("ok", "clipped", "disp", "cc"):
        np.testing.assert_array_equal(b[k], a[k], err_msg=f"{name} {k}")
    np.testing.assert_allclose(b["pce"], a["pce"], rtol=1e-12, equal_nan=True)


# one FFT-engine search in a fresh process (the pass-2 form is chosen by the environment)
_TENSOR_CHILD = r"""
import sys
import numpy as np
from pyaldvc_b200.integer_search import ncc_search
d = sys.argv[1]
z = np.load(d + "/in.npz")
sh = z["shift"] if z["shift"].any() else None
res = ncc_search(z["f"], z["g"], z["coords"], tuple(int(v) for v in z["subset"]), tuple(int(v) for v in z["radius"]), sh, engine=2)
np.savez(d + "/out.npz", **{k: np.asarray(v) for k, v in res.items()})
"""


@pytest.mark.parametrize("name", ["r16", "r9", "t15r16"])
def test_tensor_pass2_matches_reference_fft_branch(oracle_mod, gn, ncc_in, name, tmp_path):
    """ALDVC_FFT_PASS2=tensor (fft_tensor.cuh): pass 2's z transforms as tcgen05 products of TF32-split operands.
    Its FP32 maps round differently from the in-register pass, so the test holds it to the reference's FFT branch
    under the same near-tie rule as every engine, and to the in-register form: identical ok / clipped flags, integer
    peaks identical away from near ties, FP64 peak values equal where the peaks agree.  The knob is read once per
    process, so the search runs in a child process."""
    import subprocess

    from pyaldvc_b200.integer_search import ncc_search

    f, g, coords, shift = ncc_in
    c = PI.NCC_SEARCHES[name] if name in PI.NCC_SEARCHES else dict(subset=(14, 14, 14), radius=(16, 16, 16), shift=True)
    sh = shift if c["shift"] else None
    np.savez(tmp_path / "in.npz", f=f, g=g, coords=coords, subset=np.asarray(c["subset"]), radius=np.asarray(c["radius"]),
             shift=np.zeros_like(coords) if sh is None else sh)
    env = dict(os.environ, ALDVC_FFT_PASS2="tensor")
    subprocess.run([sys.executable, "-c", _TENSOR_CHILD, str(tmp_path)], env=env, check=True, timeout=900,
                   cwd=os.path.dirname(HERE))
    with np.load(tmp_path / "out.npz") as z:
        res = {k: z[k] for k in z.files}
    if name in PI.NCC_SEARCHES:
        ref = {k: gn[f"{name}_{k}"] for k in ("disp", "cc", "pce", "clipped", "ok")}
        n_ties = _compare(oracle_mod, f, g, coords, sh, c["subset"], c["radius"], res, ref, f"{name}/tensor pass 2")
        assert n_ties <= 0.02 * len(coords)
    a = ncc_search(f, g, coords, c["subset"], c["radius"], sh, engine=ENGINES["fft"])
    np.testing.assert_array_equal(res["ok"], a["ok"])
    np.testing.assert_array_equal(res["clipped"], a["clipped"])
    same = np.all(res["disp"] == a["disp"], axis=1) | ~a["ok"]
    assert (~same).sum() <= 0.01 * len(coords), f"{name}: {(~same).sum()} nodes moved against the in-register form"
    np.testing.assert_array_equal(res["cc"][same & a["ok"]], a["cc"][same & a["ok"]])


def test_fresh_process_first_search_with_a_15_voxel_template(ncc_in, tmp_path):
    """A 15^3 template at +-16 as a process's first search: the peak kernel's template and neighbour box (46.6 KB)
    plus its static shared arrays pass the 48 KB default, so the launch needs the opt-in attribute even though the
    dynamic part alone stays under it (earlier searches with larger templates used to set it in passing)."""
    import subprocess

    from pyaldvc_b200.integer_search import ncc_search

    f, g, coords, shift = ncc_in
    np.savez(tmp_path / "in.npz", f=f, g=g, coords=coords, subset=np.asarray((14, 14, 14)), radius=np.asarray((16, 16, 16)),
             shift=shift)
    subprocess.run([sys.executable, "-c", _TENSOR_CHILD, str(tmp_path)], env=dict(os.environ), check=True, timeout=900,
                   cwd=os.path.dirname(HERE))
    with np.load(tmp_path / "out.npz") as z:
        res = {k: z[k] for k in z.files}
    a = ncc_search(f, g, coords, (14, 14, 14), (16, 16, 16), shift, engine=ENGINES["fft"])
    for k in ("ok", "clipped", "disp", "cc"):
        np.testing.assert_array_equal(res[k], a[k], err_msg=k)
