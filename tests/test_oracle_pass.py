"""CPU: the oracle's whole AL-DVC pass and its FFT NCC branch against the reference's own outputs.

golden_pass.npz holds four frame pairs run through the reference's run_aldvc (core/pipeline.py:255-366, numba
backend, PCG global solver); golden_ncc_fft.npz holds integer searches where the reference's ncc_search takes
its FP32 FFT branch (integer_search.py:395, :418-443).  Both are made by tests/golden/make_golden.py.  The
fixtures store no volumes: the tests rebuild the seeded pairs (tests/golden/pass_inputs.py) and check the
SHA-256 of the oracle's normalisation against the reference-normalised volumes the fixtures were made from.
"""

from __future__ import annotations

import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))

import pass_inputs as PI  # noqa: E402


@pytest.fixture(scope="module")
def gp():
    with np.load(os.path.join(HERE, "golden", "golden_pass.npz")) as z:
        return {k: z[k] for k in z.files}


@pytest.fixture(scope="module")
def gn():
    with np.load(os.path.join(HERE, "golden", "golden_ncc_fft.npz")) as z:
        return {k: z[k] for k in z.files}


def pass_prm(name):
    """The oracle's pass parameters of a case (the reference's DVCPara names, winstepsize set by the grid)."""
    c = PI.PASS_CASES[name]
    return {k: v for k, v in c["para"].items() if k != "winstepsize"} | {"beta": PI.PASS_COMMON["beta"],
                                                                         "mu": PI.PASS_COMMON["mu"]}


def test_grid_of_the_pass_cases_is_the_reference_grid(gp):
    from pyaldvc_b200.mesh import build_grid_axes, grid_coords

    for name, c in PI.PASS_CASES.items():
        x0, y0, z0 = build_grid_axes(c["shape"], c["para"]["winsize"], c["para"]["winstepsize"])
        assert (len(z0), len(y0), len(x0)) == tuple(gp[f"{name}_grid"])
        np.testing.assert_array_equal(np.round(grid_coords(x0, y0, z0)).astype(np.int64), gp[f"{name}_coords"])


@pytest.mark.parametrize("name", list(PI.PASS_CASES))
def test_oracle_pass_matches_reference_run_aldvc(oracle_mod, gp, name):
    """Sections 3-6 of the oracle (initial guess, local 12-DOF with outlier filling, global step, ADMM with the
    reference's early stop) reproduce run_aldvc bit for bit: the same arithmetic in the same order."""
    f, g, mask, _ = PI.pass_pair(name)
    fn, gn_ = oracle_mod.normalize_volume(f), oracle_mod.normalize_volume(g)
    assert PI.sha(fn) == str(gp[f"{name}_sha_f"]) and PI.sha(gn_) == str(gp[f"{name}_sha_g"])
    o = oracle_mod.aldvc_pass(fn, gn_, gp[f"{name}_coords"], gp[f"{name}_grid"], tuple(gp[f"{name}_spacing"]), mask=mask,
                              **pass_prm(name))
    assert o["admm_steps"] == int(gp[f"{name}_steps"])
    np.testing.assert_array_equal(o["valid"], gp[f"{name}_node_valid"])
    np.testing.assert_array_equal(o["status_local"], gp[f"{name}_status_local"])
    np.testing.assert_array_equal(o["n_iter_local"], gp[f"{name}_n_iter_local"])
    np.testing.assert_array_equal(o["status"], gp[f"{name}_status"])
    np.testing.assert_array_equal(o["n_iter"], gp[f"{name}_n_iter"])
    for k in ("U0", "U_local", "F_local", "U", "F", "zncc"):
        np.testing.assert_allclose(np.asarray(o[k]).reshape(gp[f"{name}_{k}"].shape), gp[f"{name}_{k}"], rtol=0, atol=1e-12,
                                   equal_nan=True, err_msg=f"{name} {k}")


def test_pass_cases_cover_the_edge_cases(gp):
    """The fixtures hold what the parity tests lean on: early stop and forced steps, dropped nodes (mask, flat
    block), subsets that leave the volume, and the FFT branch of the search."""
    assert int(gp["affine_steps"]) < 3 and int(gp["masked_steps"]) == 3 and int(gp["fft_steps"]) == 3
    assert (~gp["masked_node_valid"]).sum() > 0 and (~gp["bspline_node_valid"]).sum() > 0
    assert (gp["fft_status"] == 2).sum() > 0
    half, rad = 8, PI.PASS_CASES["fft"]["para"]["search_radius"][0]
    assert (2 * half + 1) ** 3 * (2 * rad + 1) ** 3 > 3e7  # the reference's FFT switch


@pytest.fixture(scope="module")
def ncc_in(oracle_mod, gn):
    pair = PI.ncc_pair()
    f, g = oracle_mod.normalize_volume(pair.f), oracle_mod.normalize_volume(pair.g)
    assert PI.sha(f) == str(gn["sha_f"]) and PI.sha(g) == str(gn["sha_g"])
    coords = PI.ncc_coords()
    np.testing.assert_array_equal(coords, gn["coords"])
    np.testing.assert_array_equal(PI.ncc_shift(coords), gn["shift"])
    return f, g, coords


@pytest.mark.parametrize("name", list(PI.NCC_SEARCHES))
def test_oracle_fft_branch_matches_reference(oracle_mod, gn, ncc_in, name):
    f, g, coords = ncc_in
    c = PI.NCC_SEARCHES[name]
    res = oracle_mod.ncc_search(f, g, coords, c["subset"], c["radius"], gn["shift"] if c["shift"] else None, engine="auto")
    assert res["engine"] == "fft"
    for k in ("disp", "cc", "pce", "clipped", "ok"):
        np.testing.assert_array_equal(res[k], gn[f"{name}_{k}"], err_msg=f"{name} {k}")
    assert res["ok"].sum() > 0.9 * len(coords)


def test_oracle_fft_expansion_matches_reference(oracle_mod, gn, ncc_in):
    f, g, coords = ncc_in
    res = oracle_mod.ncc_search_expanding(f, g, coords, PI.NCC_EXPAND["subset"], PI.NCC_EXPAND["radius"], engine="auto")
    assert res["expansions"] == int(gn["expand_expansions"]) == 2
    assert tuple(res["radius"]) == tuple(gn["expand_radius"]) == (32, 32, 32)
    for k in ("disp", "cc", "pce", "clipped", "ok"):
        np.testing.assert_array_equal(res[k], gn[f"expand_{k}"], err_msg=k)


def test_oracle_window_box_stats_matches_reference(oracle_mod, gn, ncc_in):
    g = ncc_in[1]
    z, y, x = (int(v) for v in gn["box_W_origin"])
    s1, s2 = oracle_mod.window_box_stats(g[z:z + 30, y:y + 30, x:x + 30][None], 13, 11, 9)
    np.testing.assert_array_equal(s1, gn["box_sum"])
    np.testing.assert_array_equal(s2, gn["box_sq"])


def test_fft_branch_differs_from_the_exact_map_by_rounding_only(oracle_mod, gn, ncc_in):
    """The FP32 FFT map and the FP64 direct map agree to FFT rounding: the integer peaks are the same wherever
    the exact map's top two offsets are further apart than that rounding."""
    f, g, coords = ncc_in
    c = PI.NCC_SEARCHES["r16"]
    sel = np.arange(0, len(coords), 6)  # every sixth node: the FP64 direct map costs 1.8e8 multiply-adds per node
    d = oracle_mod.ncc_search(f, g, coords[sel], c["subset"], c["radius"], gn["shift"][sel], engine="direct")
    ok = gn["r16_ok"][sel]
    np.testing.assert_array_equal(d["ok"], ok)
    np.testing.assert_allclose(d["cc"][ok], gn["r16_cc"][sel][ok], rtol=0, atol=2e-6)
    np.testing.assert_allclose(d["disp"][ok], gn["r16_disp"][sel][ok], rtol=0, atol=1e-4)
