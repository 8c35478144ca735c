"""B200 kernels against the reference (golden fixtures) and against the FP64 oracle on config-sized inputs.

Parity bar (written here, taken from the reference's own GPU test test_cuda_backend.py:149-161 and the
1e-3 voxel target): identical status codes, >= 95 % identical iteration counts, |dP| < 1e-3 on converged
nodes (displacement in voxels, gradient terms dimensionless), |dZNCC| < 1e-3.  Integer NCC peaks: identical.
"""

from __future__ import annotations

import numpy as np
import pytest

from test_oracle_golden import ICGN3, ICGN12, PRE, SEARCHES, STENCIL_NOISE_GAIN, _pre_outputs, pre_args

pytestmark = pytest.mark.gpu

P_TOL = 1e-3
ZNCC_TOL = 1e-3


@pytest.fixture(scope="module")
def ck():
    from pyaldvc_b200 import cuda_kernels

    assert cuda_kernels.cuda_available(), cuda_kernels.unavailable_reason()
    return cuda_kernels


def assert_parity(ref, got, tol=P_TOL, it_frac=0.95, what=""):
    Pc, itc, stc, zc = ref
    Pg, itg, stg, zg = got
    np.testing.assert_array_equal(stg, stc, err_msg=f"{what}: status codes differ")
    assert np.mean(itc == itg) >= it_frac, f"{what}: iteration counts differ at {np.mean(itc != itg):.1%} of the nodes"
    ok = stc == 0
    if ok.any():
        assert np.max(np.abs(Pg[ok] - Pc[ok])) < tol, f"{what}: |dP| = {np.max(np.abs(Pg[ok] - Pc[ok])):.3g}"
    finite = np.isfinite(zc) & np.isfinite(zg)
    np.testing.assert_array_equal(np.isfinite(zc), np.isfinite(zg), err_msg=f"{what}: NaN pattern of zncc differs")
    if finite.any():
        assert np.max(np.abs(zg[finite] - zc[finite])) < ZNCC_TOL, what


# ----------------------------------------------------------------------------- golden fixtures (the reference's outputs)
def test_gradients_bit_exact(golden):
    import torch

    from pyaldvc_b200 import kernels as K

    gx, gy, gz = K.gradients(torch.from_numpy(golden["f"]).cuda())
    for a, k in ((gx, "gx"), (gy, "gy"), (gz, "gz")):
        np.testing.assert_array_equal(a.cpu().numpy(), golden[k])


@pytest.mark.parametrize("name", list(PRE))
def test_precompute_matches_reference(golden, ck, name):
    c, (gx, gy, gz), mask, kw = pre_args(golden, name)
    H, L, mf, bf, nv, valid = ck.precompute_nodes_cuda(golden["coords"], *c["h"], golden["f"], gx, gy, gz, mask, 0.5, 1e12,
                                                       c["stride"], **kw)
    ok = golden[f"pre_{name}_valid"]
    np.testing.assert_array_equal(valid, ok)
    np.testing.assert_array_equal(nv, golden[f"pre_{name}_n_valid"])
    Hr = golden[f"pre_{name}_H"]
    np.testing.assert_allclose(H[ok], Hr[ok], rtol=1e-4, atol=1e-5 * np.abs(Hr[ok]).max())
    np.testing.assert_allclose(mf[ok], golden[f"pre_{name}_meanf"][ok], rtol=1e-5, atol=1e-6)
    np.testing.assert_allclose(bf[ok], golden[f"pre_{name}_bottomf"][ok], rtol=1e-5)
    Lr = golden[f"pre_{name}_L"]
    np.testing.assert_allclose(L[ok], Lr[ok], rtol=1e-3, atol=1e-4 * np.abs(Lr[ok]).max())


# (variant, threads, brick_floats): brick kernel, lean kernel with 1/2/4 warps, the lean 4-warp sweep staged through TMA
# copies of g (cubic and B-spline cases with stored gradients; the others run as the lean form), plain
FORMS = [(0, 0, 0), (0, 32, 0), (0, 64, 0), (0, 128, 0), (0, 128, -1), (1, 0, 0)]
FORM_IDS = ["brick", "lean1", "lean2", "lean4", "staged", "plain"]


@pytest.mark.parametrize("form", FORMS, ids=FORM_IDS)
@pytest.mark.parametrize("name", list(ICGN12))
def test_icgn12_matches_reference(golden, ck, name, form):
    c = ICGN12[name]
    pc, (gx, gy, gz), mask, kw = pre_args(golden, c["pre"])
    H, L, mf, bf, valid = _pre_outputs(golden, c["pre"])
    g = golden["g_bspline"] if c["mode"] == 2 else golden["g"]
    P0 = golden["P0_special"] if c.get("special") else (golden["P0_far"] if c.get("far") else golden["P0"])
    gain = STENCIL_NOISE_GAIN if c.get("noise") else 0.0
    args = (golden["coords"], P0, *pc["h"], golden["f"], gx, gy, gz, mask, g, c["mode"], L, mf, bf, valid, c.get("tol", 1e-2),
            c.get("dp_tol", 1e-3), c.get("max_iter", 100), c.get("patience", 5), pc["stride"], H,
            golden[f"icgn12_{name}_pattern"], gain, c.get("predictive", True))
    got = ck.icgn_12dof_cuda(*args, **kw, variant=form[0], threads=form[1], brick_floats=form[2])
    ref = tuple(golden[f"icgn12_{name}_{k}"] for k in ("P", "n_iter", "status", "zncc"))
    assert_parity(ref, got, what=f"icgn12/{name}")
    np.testing.assert_array_equal(P0, golden["P0_special"] if c.get("special") else P0)  # P0 not mutated


@pytest.mark.parametrize("form", FORMS, ids=FORM_IDS)
@pytest.mark.parametrize("name", list(ICGN3))
def test_icgn3_matches_reference(golden, ck, name, form):
    c = ICGN3[name]
    pc, (gx, gy, gz), mask, kw = pre_args(golden, c["pre"])
    H, L, mf, bf, valid = _pre_outputs(golden, c["pre"])
    g = golden["g_bspline"] if c["mode"] == 2 else golden["g"]
    gain = STENCIL_NOISE_GAIN if c.get("noise") else 0.0
    got = ck.icgn_3dof_cuda(golden["coords"], golden["U_old"], golden["F_fixed"], golden["vdual"], *pc["h"], golden["f"], gx, gy,
                            gz, mask, g, c["mode"], H, mf, bf, valid, 1e-3, 1e-2, 1e-3, 100, 5, pc["stride"],
                            float(golden[f"icgn3_{name}_n_full"]), gain, True, **kw, variant=form[0], threads=form[1],
                            brick_floats=form[2])
    ref = tuple(golden[f"icgn3_{name}_{k}"] for k in ("U", "n_iter", "status", "zncc"))
    assert_parity(ref, got, what=f"icgn3/{name}")


def test_chunked_launches_match_one_launch(golden, ck):
    c, (gx, gy, gz), mask, kw = pre_args(golden, "plain")
    H, L, mf, bf, valid = _pre_outputs(golden, "plain")
    args = (golden["coords"], golden["P0"], *c["h"], golden["f"], gx, gy, gz, mask, golden["g"], 1, L, mf, bf, valid, 1e-2, 1e-3,
            100, 5)
    full = ck.icgn_12dof_cuda(*args)
    seen = []
    part = ck.icgn_12dof_cuda(*args, chunk=7, progress_fn=seen.append)
    for a, b in zip(full, part):
        np.testing.assert_array_equal(a, b)
    assert seen and seen[-1] == 1.0 and len(seen) >= 2


def test_zncc_map_matches_reference(golden, ck):
    hx, hy, hz = (int(a) for a in golden["zncc_h"])
    rx, ry, rz = (int(a) for a in golden["zncc_r"])
    ref = golden["zncc_map"]
    out = np.empty_like(ref)
    ck.zncc_direct_cuda(golden["f"], golden["g"], golden["coords"], hx, hy, hz, rx, ry, rz, golden["zncc_wx0"], golden["zncc_wy0"],
                        golden["zncc_wz0"], golden["zncc_t_ok"], out)
    np.testing.assert_allclose(out, ref, rtol=0, atol=2e-5)
    flat = np.ones_like(golden["f"])
    out2 = np.empty_like(golden["zncc_map_flat"])
    ck.zncc_direct_cuda(flat, golden["g"], golden["coords"][:2], hx, hy, hz, rx, ry, rz, golden["zncc_wx0"][:2],
                        golden["zncc_wy0"][:2], golden["zncc_wz0"][:2], np.ones(2, bool), out2)
    np.testing.assert_array_equal(out2, golden["zncc_map_flat"])


def _check_search(res, ref_get, name):
    np.testing.assert_array_equal(res["ok"], ref_get("ok"), err_msg=name)
    np.testing.assert_array_equal(res["clipped"], ref_get("clipped"), err_msg=name)
    d, dr = res["disp"], ref_get("disp")
    ok = ref_get("ok")
    # integer peak identical: the integer part of disp is the peak offset (sub-voxel part is in (-1, 1))
    np.testing.assert_allclose(d[ok], dr[ok], rtol=0, atol=1e-6, err_msg=name)
    np.testing.assert_allclose(res["cc"][ok], ref_get("cc")[ok], rtol=0, atol=1e-9, err_msg=name)
    np.testing.assert_allclose(res["pce"][ok], ref_get("pce")[ok], rtol=1e-3, err_msg=name)


@pytest.mark.parametrize("engine", [0, 1, 2], ids=["tiled", "plain", "fft"])
@pytest.mark.parametrize("name", list(SEARCHES))
def test_ncc_search_matches_reference(golden, name, engine):
    from pyaldvc_b200.integer_search import ncc_search

    c = SEARCHES[name]
    shift = np.round(golden["U_true"]).astype(np.int64) if c["shift"] else None
    res = ncc_search(golden["f"], golden["g"], golden["coords"], c["subset"], c["radius"], shift, engine=engine)
    _check_search(res, lambda k: golden[f"ncc_{name}_{k}"], name)


@pytest.mark.parametrize("engine", [0, 1, 2], ids=["tiled", "plain", "fft"])
def test_ncc_search_expanding_matches_reference(golden, engine):
    from pyaldvc_b200.integer_search import ncc_search_expanding

    res = ncc_search_expanding(golden["f"], golden["g"], golden["coords"], (8, 8, 8), (1, 1, 1), engine=engine)
    assert res["expansions"] == int(golden["nccx_expansions"])
    _check_search(res, lambda k: golden[f"nccx_{k}"], "expanding")


def test_global_step_matches_reference(golden):
    from pyaldvc_b200.subpb2_solver import HexGrid, build_global_system, global_rhs, nodal_gradient, solve_subpb2

    grid = HexGrid(tuple(int(s) for s in golden["pcg_grid_shape"]), tuple(float(s) for s in golden["pcg_spacing"]),
                   golden["pcg_elem_active"])
    system = build_global_system(grid, 1e-3, 1e-3, 0.0, pcg_tol=1e-10)
    args = (golden["pcg_U1"], golden["pcg_F1"], golden["pcg_W"], golden["pcg_v"])
    np.testing.assert_allclose(global_rhs(system, *args), golden["pcg_rhs"], rtol=1e-11, atol=1e-14)
    U2, info = solve_subpb2(system, *args)
    assert abs(info["iterations"] - int(golden["pcg_iters"])) <= 1
    np.testing.assert_allclose(U2, golden["pcg_U2"], rtol=0, atol=1e-8)
    F = nodal_gradient(system, U2)
    np.testing.assert_allclose(F, golden["pcg_F"], rtol=0, atol=1e-8, equal_nan=True)
    system2 = build_global_system(grid, 0.05, 1e-3, 0.01, pcg_tol=1e-10)
    U2b, info2 = solve_subpb2(system2, *args)
    assert abs(info2["iterations"] - int(golden["pcg_alpha_iters"])) <= 1
    np.testing.assert_allclose(U2b, golden["pcg_alpha_U2"], rtol=0, atol=1e-8)


@pytest.fixture(scope="module")
def config1_pair():
    from pyaldvc_b200 import configs, synthetic
    from pyaldvc_b200.mesh import build_grid_axes, grid_coords

    pair = configs.host_pair(1)
    f = synthetic.normalize_volume(pair.f)
    g = synthetic.normalize_volume(pair.g)
    x0, y0, z0 = build_grid_axes(f.shape, (20, 20, 20), (8, 8, 8))
    coords = np.round(grid_coords(x0, y0, z0)).astype(np.int64)
    return f, g, coords


@pytest.mark.parametrize("engine", [0, 1, 2], ids=["tiled", "plain", "fft"])
@pytest.mark.parametrize("radius", [4, 8])
def test_ncc_search_17cube_template_matches_oracle(oracle_mod, config1_pair, engine, radius):
    """Default template of the pipeline (17^3, min(winsize, 16)) against the FP64 direct map of the oracle."""
    from pyaldvc_b200.integer_search import ncc_search

    f, g, coords = config1_pair
    ref = oracle_mod.ncc_search(f, g, coords, (16, 16, 16), (radius,) * 3)
    res = ncc_search(f, g, coords, (16, 16, 16), (radius,) * 3, engine=engine)
    _check_search(res, lambda k: ref[k], f"17^3 r{radius}")


@pytest.fixture(scope="module")
def bead_pair_100():
    from pyaldvc_b200 import synthetic as S

    shape = (100, 100, 100)
    c, pk = S.draw_beads(shape, 0.03, 21)
    f = S.normalize_volume(S.render_beads(shape, c, pk, 1.5))
    g = S.normalize_volume(S.render_beads(shape, S.displace_beads(c, S.translation((2.6, -5.3, 7.4))), pk, 1.5))
    ax = np.arange(20, 81, 12)
    zz, yy, xx = np.meshgrid(ax, ax, ax, indexing="ij")
    return f, g, np.stack([xx.ravel(), yy.ravel(), zz.ravel()], 1).astype(np.int64)


@pytest.mark.parametrize("engine", [2, 3], ids=["fft", "fft_stockham"])
@pytest.mark.parametrize("radius", [4, 8, 16, 32])
def test_ncc_fft_engine_matches_tiled_engine_at_large_radius(bead_pair_100, radius, engine):
    """The FFT engine (in-register transforms where the box is cubic with a compiled length -- 36 at +-8, 50 at
    +-16 -- and Stockham transforms elsewhere; engine 3 forces Stockham everywhere) against the tiled direct engine
    at the +-16 search of the 1024^2 x 306 workload, its first expansion (+-32, 81-voxel windows) and small radii:
    identical integer peaks, ok/clipped flags and FP64 re-scored cc."""
    from pyaldvc_b200.integer_search import ncc_search

    f, g, coords = bead_pair_100
    a = ncc_search(f, g, coords, (16, 16, 16), (radius,) * 3, engine=0)
    b = ncc_search(f, g, coords, (16, 16, 16), (radius,) * 3, engine=engine)
    assert a["ok"].sum() > 100
    _check_search(b, lambda k: a[k], f"fft vs tiled r{radius}")
