"""The CPU oracle against the reference's own outputs (tests/golden, made by make_golden.py).

Both sides compute in FP64 with the same loop order, so the bar is ~1e-10 and
identical status codes / iteration counts.
"""

from __future__ import annotations

import numpy as np
import pytest

PRE = {
    "plain": dict(h=(5, 5, 5), stride=1, grads="stored", mask=False, split=False),
    "aniso": dict(h=(4, 5, 6), stride=1, grads="stored", mask=False, split=False),
    "masked": dict(h=(5, 5, 5), stride=1, grads="stored", mask=True, split=False),
    "stride2": dict(h=(5, 5, 5), stride=2, grads="stored", mask=False, split=False),
    "otf": dict(h=(5, 5, 5), stride=1, grads="otf", mask=False, split=False),
    "split": dict(h=(5, 5, 5), stride=1, grads="stored", mask=True, split=True),
}
ICGN12 = {
    "cubic": dict(pre="plain", mode=1),
    "linear": dict(pre="plain", mode=0),
    "bspline": dict(pre="plain", mode=2),
    "aniso": dict(pre="aniso", mode=1),
    "masked": dict(pre="masked", mode=1),
    "stride2": dict(pre="stride2", mode=1),
    "otf": dict(pre="otf", mode=1),
    "split": dict(pre="split", mode=1),
    "noise": dict(pre="plain", mode=1, noise=True),
    "nopredict": dict(pre="plain", mode=1, predictive=False),
    "special": dict(pre="plain", mode=1, special=True),
    "stall": dict(pre="plain", mode=1, patience=1, far=True),
    "maxiter": dict(pre="plain", mode=1, max_iter=2, tol=1e-9, dp_tol=1e-12, patience=0),
}
ICGN3 = {
    "cubic": dict(pre="plain", mode=1),
    "linear": dict(pre="plain", mode=0),
    "masked": dict(pre="masked", mode=1),
    "noise": dict(pre="plain", mode=1, noise=True),
    "split": dict(pre="split", mode=1),
    "stride2": dict(pre="stride2", mode=2),
}
STENCIL_NOISE_GAIN = float(np.sum(np.array([-1 / 60, 3 / 20, -3 / 4, 0.0, 3 / 4, -3 / 20, 1 / 60]) ** 2))


def pre_args(gd, name):
    c = PRE[name]
    ph = np.zeros((1, 1, 1), np.float32)
    grads = (gd["gx"], gd["gy"], gd["gz"]) if c["grads"] == "stored" else (ph, ph, ph)
    mask = gd["mask"] if c["mask"] else np.ones((1, 1, 1), np.uint8)
    kw = {"split_index": gd["split_index"], "split_keep": gd["split_keep"]} if c["split"] else {}
    return c, grads, mask, kw


def test_interp_matches_reference(golden, oracle_mod):
    for mode in (0, 1, 2):
        src = golden["f_bspline"] if mode == 2 else golden["f"]
        got = oracle_mod.sample_points(src, golden["pts_z"], golden["pts_y"], golden["pts_x"], mode)
        np.testing.assert_allclose(got, golden[f"interp_{mode}"], rtol=0, atol=1e-12, equal_nan=True)
    assert np.isnan(golden["interp_1"]).any()  # points outside the admissible domain stay NaN


def test_gradients_match_reference(golden, oracle_mod):
    gx, gy, gz = oracle_mod.compute_gradients(golden["f"])
    for a, k in ((gx, "gx"), (gy, "gy"), (gz, "gz")):
        np.testing.assert_array_equal(a, golden[k])


def test_compose_warp_matches_reference(golden, oracle_mod):
    P, ok = oracle_mod.compose_warp(golden["compose_P"], golden["compose_dP"])
    assert ok
    np.testing.assert_allclose(P, golden["compose_out"], atol=1e-15)


@pytest.mark.parametrize("name", list(PRE))
def test_precompute_matches_reference(golden, oracle_mod, name):
    c, (gx, gy, gz), mask, kw = pre_args(golden, name)
    H, L, mf, bf, nv, valid = oracle_mod.precompute_nodes(golden["coords"], *c["h"], golden["f"], gx, gy, gz, mask, 0.5, 1e12,
                                                          c["stride"], **kw)
    np.testing.assert_array_equal(valid, golden[f"pre_{name}_valid"])
    np.testing.assert_array_equal(nv, golden[f"pre_{name}_n_valid"])
    np.testing.assert_allclose(H, golden[f"pre_{name}_H"], rtol=1e-12, atol=1e-9)
    np.testing.assert_allclose(L, golden[f"pre_{name}_L"], rtol=1e-10, atol=1e-9)
    np.testing.assert_allclose(mf, golden[f"pre_{name}_meanf"], rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(bf, golden[f"pre_{name}_bottomf"], rtol=1e-12, atol=1e-12)


def _pre_outputs(gd, name):
    return (gd[f"pre_{name}_H"], gd[f"pre_{name}_L"], gd[f"pre_{name}_meanf"], gd[f"pre_{name}_bottomf"],
            gd[f"pre_{name}_valid"])


@pytest.mark.parametrize("name", list(ICGN12))
def test_icgn12_matches_reference(golden, oracle_mod, name):
    c = ICGN12[name]
    pc, (gx, gy, gz), mask, kw = pre_args(golden, c["pre"])
    H, L, mf, bf, valid = _pre_outputs(golden, c["pre"])
    g = golden["g_bspline"] if c["mode"] == 2 else golden["g"]
    P0 = golden["P0_special"] if c.get("special") else (golden["P0_far"] if c.get("far") else golden["P0"])
    gain = STENCIL_NOISE_GAIN if c.get("noise") else 0.0
    P, it, st, zc = oracle_mod.icgn_12dof_parallel(
        golden["coords"], P0, *pc["h"], golden["f"], gx, gy, gz, mask, g, c["mode"], L, mf, bf, valid, c.get("tol", 1e-2),
        c.get("dp_tol", 1e-3), c.get("max_iter", 100), c.get("patience", 5), pc["stride"], H, golden[f"icgn12_{name}_pattern"],
        gain, c.get("predictive", True), **kw)
    np.testing.assert_array_equal(st, golden[f"icgn12_{name}_status"])
    np.testing.assert_array_equal(it, golden[f"icgn12_{name}_n_iter"])
    np.testing.assert_allclose(P, golden[f"icgn12_{name}_P"], rtol=0, atol=1e-10, equal_nan=True)
    np.testing.assert_allclose(zc, golden[f"icgn12_{name}_zncc"], rtol=0, atol=1e-10, equal_nan=True)


def test_icgn12_golden_cases_exercise_statuses(golden):
    assert (golden["icgn12_cubic_status"] == 0).mean() > 0.9
    sp = golden["icgn12_special_status"]
    assert sp[0] == 5 and sp[1] == 2
    assert (golden["icgn12_stall_status"] == 7).any()
    assert (golden["icgn12_maxiter_status"] == 1).any()
    assert (golden["icgn12_masked_status"] == 3).any()


@pytest.mark.parametrize("name", list(ICGN3))
def test_icgn3_matches_reference(golden, oracle_mod, name):
    c = ICGN3[name]
    pc, (gx, gy, gz), mask, kw = pre_args(golden, c["pre"])
    H, L, mf, bf, valid = _pre_outputs(golden, c["pre"])
    g = golden["g_bspline"] if c["mode"] == 2 else golden["g"]
    gain = STENCIL_NOISE_GAIN if c.get("noise") else 0.0
    U, it, st, zc = oracle_mod.icgn_3dof_parallel(
        golden["coords"], golden["U_old"], golden["F_fixed"], golden["vdual"], *pc["h"], golden["f"], gx, gy, gz, mask, g,
        c["mode"], H, mf, bf, valid, 1e-3, 1e-2, 1e-3, 100, 5, pc["stride"], float(golden[f"icgn3_{name}_n_full"]), gain, True,
        **kw)
    np.testing.assert_array_equal(st, golden[f"icgn3_{name}_status"])
    np.testing.assert_array_equal(it, golden[f"icgn3_{name}_n_iter"])
    np.testing.assert_allclose(U, golden[f"icgn3_{name}_U"], rtol=0, atol=1e-10, equal_nan=True)
    np.testing.assert_allclose(zc, golden[f"icgn3_{name}_zncc"], rtol=0, atol=1e-10, equal_nan=True)


def test_zncc_direct_matches_reference(golden, oracle_mod):
    hx, hy, hz = (int(a) for a in golden["zncc_h"])
    rx, ry, rz = (int(a) for a in golden["zncc_r"])
    ref = golden["zncc_map"]
    out = np.empty_like(ref)
    oracle_mod.zncc_direct(golden["f"], golden["g"], golden["coords"], hx, hy, hz, rx, ry, rz, golden["zncc_wx0"],
                           golden["zncc_wy0"], golden["zncc_wz0"], golden["zncc_t_ok"], out)
    np.testing.assert_allclose(out, ref, rtol=0, atol=1e-12)
    flat = np.ones_like(golden["f"])
    out2 = np.empty_like(golden["zncc_map_flat"])
    oracle_mod.zncc_direct(flat, golden["g"], golden["coords"][:2], hx, hy, hz, rx, ry, rz, golden["zncc_wx0"][:2],
                           golden["zncc_wy0"][:2], golden["zncc_wz0"][:2], np.ones(2, bool), out2)
    np.testing.assert_array_equal(out2, golden["zncc_map_flat"])


SEARCHES = {
    "r3": dict(subset=(8, 8, 8), radius=(3, 3, 3), shift=False),
    "shift": dict(subset=(8, 8, 8), radius=(2, 2, 2), shift=True),
    "aniso": dict(subset=(6, 8, 10), radius=(3, 2, 1), shift=False),
    "r1": dict(subset=(8, 8, 8), radius=(1, 1, 1), shift=False),
}


@pytest.mark.parametrize("name", list(SEARCHES))
def test_ncc_search_matches_reference(golden, oracle_mod, name):
    c = SEARCHES[name]
    shift = np.round(golden["U_true"]).astype(np.int64) if c["shift"] else None
    res = oracle_mod.ncc_search(golden["f"], golden["g"], golden["coords"], c["subset"], c["radius"], shift)
    np.testing.assert_array_equal(res["ok"], golden[f"ncc_{name}_ok"])
    np.testing.assert_array_equal(res["clipped"], golden[f"ncc_{name}_clipped"])
    np.testing.assert_allclose(res["disp"], golden[f"ncc_{name}_disp"], atol=1e-9, equal_nan=True)
    np.testing.assert_allclose(res["cc"], golden[f"ncc_{name}_cc"], atol=1e-12, equal_nan=True)
    np.testing.assert_allclose(res["pce"], golden[f"ncc_{name}_pce"], rtol=1e-9, equal_nan=True)


def test_ncc_search_expanding_matches_reference(golden, oracle_mod):
    res = oracle_mod.ncc_search_expanding(golden["f"], golden["g"], golden["coords"], (8, 8, 8), (1, 1, 1))
    assert res["expansions"] == int(golden["nccx_expansions"])
    assert tuple(res["radius"]) == tuple(golden["nccx_radius"])
    np.testing.assert_array_equal(res["ok"], golden["nccx_ok"])
    np.testing.assert_allclose(res["disp"], golden["nccx_disp"], atol=1e-9, equal_nan=True)


def _pcg_ops(gd, oracle_mod):
    return oracle_mod.fem_operators(tuple(gd["pcg_grid_shape"]), tuple(gd["pcg_spacing"]), gd["pcg_elem_active"])


def test_global_step_matches_reference(golden, oracle_mod):
    ops = _pcg_ops(golden, oracle_mod)
    np.testing.assert_array_equal(ops["active"], golden["pcg_active"])
    b = oracle_mod.global_rhs(ops, 1e-3, 1e-3, 0.0, golden["pcg_U1"], golden["pcg_F1"], golden["pcg_W"], golden["pcg_v"])
    np.testing.assert_allclose(b, golden["pcg_rhs"], rtol=1e-12, atol=1e-14)
    system = oracle_mod.global_system(ops, 1e-3, 1e-3, 0.0)
    U2, it = oracle_mod.solve_subpb2(system, golden["pcg_U1"], golden["pcg_F1"], golden["pcg_W"], golden["pcg_v"], tol=1e-10)
    assert it == int(golden["pcg_iters"])
    np.testing.assert_allclose(U2, golden["pcg_U2"], rtol=0, atol=1e-10)
    F = oracle_mod.nodal_gradient(ops, U2)
    np.testing.assert_allclose(F, golden["pcg_F"], rtol=0, atol=1e-10, equal_nan=True)
    system2 = oracle_mod.global_system(ops, 0.05, 1e-3, 0.01)
    U2b, itb = oracle_mod.solve_subpb2(system2, golden["pcg_U1"], golden["pcg_F1"], golden["pcg_W"], golden["pcg_v"], tol=1e-10)
    assert itb == int(golden["pcg_alpha_iters"])
    np.testing.assert_allclose(U2b, golden["pcg_alpha_U2"], rtol=0, atol=1e-10)
