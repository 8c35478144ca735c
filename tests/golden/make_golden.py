"""Generate the golden fixtures that pin the CPU oracle to the reference.

Run in a container that holds the pyALDVC sources (read-only) at
``$ALDVC_REFERENCE/src`` (default ``/root/reference/src``)::

    NUMBA_CACHE_DIR=/tmp/numba_cache python tests/golden/make_golden.py [kernels volume_ops init_guess strain beta pass ncc_fft tiling series]

It imports the reference package, runs its own Numba CPU kernels on seeded
bead volumes from ``pyaldvc_b200.synthetic`` and stores inputs + outputs as
small ``.npz`` files next to this script.  The tests only read the fixtures;
nothing at test time needs the reference.
"""

from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)
sys.path.insert(0, os.path.join(os.environ.get("ALDVC_REFERENCE", "/root/reference"), "src"))
os.environ.setdefault("NUMBA_CACHE_DIR", "/tmp/numba_cache")

from al_dvc.core.config import dvcpara_default  # noqa: E402
from al_dvc.core.data_structures import P_from_UF  # noqa: E402
from al_dvc.io.volume_ops import compute_gradients, normalize_volume, prefilter_bspline, presmooth_volume  # noqa: E402
from al_dvc.mesh.grid_mesh import build_grid_axes as ref_grid_axes  # noqa: E402
from al_dvc.mesh.grid_mesh import mesh_setup  # noqa: E402
from al_dvc.solver import integer_search as ris  # noqa: E402
from al_dvc.solver import numba_kernels as nk  # noqa: E402
from al_dvc.solver.global_operators import build_fem_operators, nodal_gradient  # noqa: E402
from al_dvc.solver.interp_kernels import sample_points  # noqa: E402
from al_dvc.solver.subpb2_solver import build_global_system, global_rhs, solve_subpb2  # noqa: E402
from al_dvc.solver.uncertainty import STENCIL_NOISE_GAIN, noise_hessian_pattern  # noqa: E402

from pyaldvc_b200 import synthetic as syn  # noqa: E402

sys.path.insert(0, HERE)
import init_guess_inputs as IG  # noqa: E402

SHAPE = (32, 34, 36)  # (nz, ny, nx), non-cubic on purpose
F_TRUE = np.array([[0.015, 0.004, 0.0], [0.003, -0.01, 0.002], [0.0, -0.002, 0.012]])
T_TRUE = (1.3, -0.7, 0.4)
CENTRE = ((SHAPE[2] - 1) / 2, (SHAPE[1] - 1) / 2, (SHAPE[0] - 1) / 2)


def volumes():
    disp = syn.affine(F_TRUE, T_TRUE, CENTRE)
    pair = syn.bead_pair(SHAPE, density=0.03, sigma=1.5, seed=11, disp=disp, noise=0.01)
    f = normalize_volume(pair.f)
    g = normalize_volume(pair.g)
    return f, g, disp


def main():
    f, g, disp = volumes()
    gx, gy, gz = compute_gradients(f)
    g_bs = prefilter_bspline(g)
    f_bs = prefilter_bspline(f)
    out = {"f": f, "g": g, "gx": gx, "gy": gy, "gz": gz, "g_bspline": g_bs, "f_bspline": f_bs}

    # --- interpolation (interp_kernels.sample_points) ---
    rng = np.random.default_rng(0)
    npts = 300
    zs = rng.uniform(0.5, SHAPE[0] - 2.5, npts)
    ys = rng.uniform(0.5, SHAPE[1] - 2.5, npts)
    xs = rng.uniform(0.5, SHAPE[2] - 2.5, npts)
    out.update(pts_z=zs, pts_y=ys, pts_x=xs)
    for mode in (0, 1, 2):
        src = f_bs if mode == 2 else f
        out[f"interp_{mode}"] = sample_points(src, zs, ys, xs, mode)

    # --- warp composition ---
    Pc = rng.normal(0, 0.05, 12)
    dPc = rng.normal(0, 0.02, 12)
    P1 = Pc.copy()
    nk.compose_warp_inplace(P1, dPc)
    out.update(compose_P=Pc, compose_dP=dPc, compose_out=P1)

    # --- node grid (winsize 10, step 6) ---
    x0, y0, z0 = ref_grid_axes(dvcpara_default().voi, SHAPE, (10, 10, 10), (6, 6, 6))
    mesh = mesh_setup(x0, y0, z0)
    coords = np.round(mesh.coordinates).astype(np.int64)
    out.update(coords=coords, grid_shape=np.array(mesh.grid_shape), x0=x0, y0=y0, z0=z0)
    N = coords.shape[0]
    U_true = np.column_stack(disp(coords[:, 0].astype(float), coords[:, 1].astype(float), coords[:, 2].astype(float)))
    out["U_true"] = U_true

    mask = np.ones(SHAPE, dtype=np.uint8)
    mask[:, :, 20:] = 0  # a slab of non-material: the last node column loses its subsets
    out["mask"] = mask
    placeholder = np.zeros((1, 1, 1), dtype=np.float32)
    nomask = np.ones((1, 1, 1), dtype=np.uint8)

    # split rows for the masked case (subset splitting)
    cand = np.arange(N)
    rows, n_keep, n_inmask = nk.build_split_rows(coords, cand, 5, 5, 5, 1, mask, 0)
    split_index = np.arange(N, dtype=np.int64)
    out.update(split_keep=rows, split_index=split_index)

    pre_cases = {
        "plain": dict(h=(5, 5, 5), stride=1, grads="stored", mask=False, split=False),
        "aniso": dict(h=(4, 5, 6), stride=1, grads="stored", mask=False, split=False),
        "masked": dict(h=(5, 5, 5), stride=1, grads="stored", mask=True, split=False),
        "stride2": dict(h=(5, 5, 5), stride=2, grads="stored", mask=False, split=False),
        "otf": dict(h=(5, 5, 5), stride=1, grads="otf", mask=False, split=False),
        "split": dict(h=(5, 5, 5), stride=1, grads="stored", mask=True, split=True),
    }
    contexts = {}
    for name, c in pre_cases.items():
        hx, hy, hz = c["h"]
        gxa, gya, gza = (gx, gy, gz) if c["grads"] == "stored" else (placeholder,) * 3
        m = mask if c["mask"] else nomask
        kw = {"split_index": split_index, "split_keep": rows} if c["split"] else {}
        H, L, mf, bf, nv, valid = nk.precompute_nodes(coords, hx, hy, hz, f, gxa, gya, gza, m, 0.5, 1e12, c["stride"], **kw)
        for k, v in zip(("H", "L", "meanf", "bottomf", "n_valid", "valid"), (H, L, mf, bf, nv, valid)):
            out[f"pre_{name}_{k}"] = v
        contexts[name] = (c, gxa, gya, gza, m, kw, H, L, mf, bf, valid)

    # --- 12-DOF IC-GN ---
    P0 = P_from_UF(np.round(U_true) + np.array([0.2, -0.1, 0.15]), np.zeros((N, 3, 3)))
    P0_special = P0.copy()
    P0_special[0, 9] = np.nan  # NaN start -> status 5
    P0_special[1, 9] = 60.0  # warps outside the volume -> status 2
    P0_far = P0.copy()
    P0_far[:, 9:] = np.round(U_true) + np.array([3.5, -3.5, 2.45])  # far start: some nodes stall, some leave the volume
    out["P0"] = P0
    out["P0_special"] = P0_special
    out["P0_far"] = P0_far
    icgn_cases = {
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
    for name, c in icgn_cases.items():
        cc, gxa, gya, gza, m, kw, H, L, mf, bf, valid = contexts[c["pre"]]
        hx, hy, hz = cc["h"]
        gsrc = g_bs if c["mode"] == 2 else g
        pattern = noise_hessian_pattern((hx, hy, hz), cc["stride"])
        gain = STENCIL_NOISE_GAIN if c.get("noise") else 0.0
        P_start = P0_special if c.get("special") else (P0_far if c.get("far") else P0)
        res = nk.icgn_12dof_parallel(coords, P_start.copy(), hx, hy, hz, f, gxa, gya, gza, m, gsrc, c["mode"], L, mf, bf, valid,
                                     c.get("tol", 1e-2), c.get("dp_tol", 1e-3), c.get("max_iter", 100), c.get("patience", 5),
                                     cc["stride"], H, pattern, gain, c.get("predictive", True), **kw)
        for k, v in zip(("P", "n_iter", "status", "zncc"), res):
            out[f"icgn12_{name}_{k}"] = v
        out[f"icgn12_{name}_pattern"] = pattern

    # --- 3-DOF IC-GN (ADMM subproblem 1) ---
    U_old = U_true + np.array([0.25, -0.2, 0.15])
    F_fixed = np.tile(F_TRUE, (N, 1, 1))
    vdual = np.column_stack([0.02 * np.sin(np.arange(N)), 0.01 * np.cos(np.arange(N)), np.zeros(N)])
    out.update(U_old=U_old, F_fixed=F_fixed, vdual=vdual)
    icgn3_cases = {
        "cubic": dict(pre="plain", mode=1),
        "linear": dict(pre="plain", mode=0),
        "masked": dict(pre="masked", mode=1),
        "noise": dict(pre="plain", mode=1, noise=True),
        "split": dict(pre="split", mode=1),
        "stride2": dict(pre="stride2", mode=2),
    }
    for name, c in icgn3_cases.items():
        cc, gxa, gya, gza, m, kw, H, L, mf, bf, valid = contexts[c["pre"]]
        hx, hy, hz = cc["h"]
        gsrc = g_bs if c["mode"] == 2 else g
        pattern = noise_hessian_pattern((hx, hy, hz), cc["stride"])
        gain = STENCIL_NOISE_GAIN if c.get("noise") else 0.0
        res = nk.icgn_3dof_parallel(coords, U_old, F_fixed, vdual, hx, hy, hz, f, gxa, gya, gza, m, gsrc, c["mode"], H, mf, bf, valid,
                                    1e-3, 1e-2, 1e-3, 100, 5, cc["stride"], float(pattern[9, 9]), gain, True, **kw)
        for k, v in zip(("U", "n_iter", "status", "zncc"), res):
            out[f"icgn3_{name}_{k}"] = v
        out[f"icgn3_{name}_n_full"] = float(pattern[9, 9])

    # --- integer search ---
    hx = hy = hz = 4
    rx, ry, rz = 3, 2, 3
    sx, sy, sz = 2 * hx + 1, 2 * hy + 1, 2 * hz + 1
    wx, wy, wz = sx + 2 * rx, sy + 2 * ry, sz + 2 * rz
    wx0 = np.clip(coords[:, 0] + 1 - hx - rx, 0, SHAPE[2] - wx)
    wy0 = np.clip(coords[:, 1] - 1 - hy - ry, 0, SHAPE[1] - wy)
    wz0 = np.clip(coords[:, 2] - hz - rz, 0, SHAPE[0] - wz)
    t_ok = np.ones(N, dtype=np.bool_)
    t_ok[3] = False
    zmap = np.empty((N, 2 * rz + 1, 2 * ry + 1, 2 * rx + 1))
    ris._zncc_direct(f, g, coords, hx, hy, hz, rx, ry, rz, wx0, wy0, wz0, t_ok, zmap)
    out.update(zncc_map=zmap, zncc_wx0=wx0, zncc_wy0=wy0, zncc_wz0=wz0, zncc_t_ok=t_ok, zncc_h=np.array([hx, hy, hz]),
               zncc_r=np.array([rx, ry, rz]))
    flat = f.copy()
    flat[:, :, :] = 1.0  # flat template -> map of -2, never ok
    zmap_flat = np.empty((2, 2 * rz + 1, 2 * ry + 1, 2 * rx + 1))
    ris._zncc_direct(flat, g, coords[:2], hx, hy, hz, rx, ry, rz, wx0[:2], wy0[:2], wz0[:2], np.ones(2, bool), zmap_flat)
    out["zncc_map_flat"] = zmap_flat

    searches = {
        "r3": dict(subset=(8, 8, 8), radius=(3, 3, 3), shift=None),
        "shift": dict(subset=(8, 8, 8), radius=(2, 2, 2), shift=np.round(U_true).astype(np.int64)),
        "aniso": dict(subset=(6, 8, 10), radius=(3, 2, 1), shift=None),
        "r1": dict(subset=(8, 8, 8), radius=(1, 1, 1), shift=None),
    }
    for name, c in searches.items():
        res = ris.ncc_search(f, g, coords, c["subset"], c["radius"], c["shift"], backend="numba")
        for k in ("disp", "cc", "pce", "clipped", "ok"):
            out[f"ncc_{name}_{k}"] = res[k]
    res = ris.ncc_search_expanding(f, g, coords, (8, 8, 8), (1, 1, 1), None, True, 3, backend="numba")
    for k in ("disp", "cc", "pce", "clipped", "ok"):
        out[f"nccx_{k}"] = res[k]
    out["nccx_expansions"] = res["expansions"]
    out["nccx_radius"] = np.array(res["radius"])

    # --- global step (hex8 FEM, PCG) ---
    gm = mesh_setup(np.arange(6) * 6.0, np.arange(5) * 7.0, np.arange(4) * 5.0)
    nn = gm.n_nodes
    node_valid = np.ones(nn, dtype=bool)
    node_valid[[7, 8, 33]] = False
    elems = gm.elements.copy()
    bad = ~node_valid[elems].all(axis=1)
    elems[bad, :] = -1
    gm.elements = elems
    gm.node_valid = node_valid
    ops = build_fem_operators(gm, 2)
    para = dvcpara_default(global_solver="pcg", pcg_tol=1e-10, pcg_max_iter=500)
    rng = np.random.default_rng(5)
    U1 = rng.normal(0, 0.5, (nn, 3))
    F1 = rng.normal(0, 0.01, (nn, 3, 3))
    W = rng.normal(0, 0.002, (nn, 3, 3))
    v = rng.normal(0, 0.05, (nn, 3))
    system = build_global_system(ops, 1e-3, 1e-3, 0.0, para)
    U2, info = solve_subpb2(system, U1, F1, W, v)
    Fg = nodal_gradient(ops, U2)
    b = global_rhs(ops, 1e-3, 1e-3, 0.0, U1, F1, W, v)
    out.update(pcg_elem_active=~bad, pcg_grid_shape=np.array(gm.grid_shape), pcg_spacing=np.array(gm.spacing), pcg_U1=U1,
               pcg_F1=F1, pcg_W=W, pcg_v=v, pcg_U2=U2, pcg_iters=info["iterations"], pcg_F=Fg, pcg_rhs=b,
               pcg_active=ops.active)
    system2 = build_global_system(ops, 0.05, 1e-3, 0.01, para)
    U2b, infob = solve_subpb2(system2, U1, F1, W, v)
    out.update(pcg_alpha_U2=U2b, pcg_alpha_iters=infob["iterations"])

    path = os.path.join(HERE, "golden_kernels.npz")
    np.savez_compressed(path, **out)
    print(f"wrote {path} ({os.path.getsize(path) / 1e6:.2f} MB)")


def volume_ops_fixtures():
    """The reference's whole-volume filters on a bead volume whose x lines are longer than one device tile (197)
    and whose z lines are short (10), plus a 5 x 3 x 2 volume of lines of 1, 2, 3 and 5 samples."""
    shape = (10, 17, 197)
    pair = syn.bead_pair(shape, density=0.03, sigma=1.5, seed=21, disp=syn.translation((0.0, 0.0, 0.0)), noise=0.01)
    v = normalize_volume(pair.f)
    small = np.random.default_rng(22).normal(0.0, 1.0, (5, 3, 2)).astype(np.float32)
    from al_dvc.core.data_structures import VOIRange

    raw = np.random.default_rng(23).integers(0, 4096, (12, 20, 45)).astype(np.uint16)
    raw[3:9, 5:15, 10:30] += 200  # a brighter block, so the VOI statistics differ from the whole volume's
    out = {"norm_raw": raw, "norm_whole": normalize_volume(raw),
           "norm_voi": normalize_volume(raw, VOIRange(x=(8, 33), y=(4, 16), z=(2, 10))),
           "vol": v, "bspline": prefilter_bspline(v), "gauss_0.8": presmooth_volume(v, 0.8),
           "gauss_2.0": presmooth_volume(v, 2.0), "small": small, "small_bspline": prefilter_bspline(small),
           "small_gauss_1.0": presmooth_volume(small, 1.0)}
    path = os.path.join(HERE, "golden_volume_ops.npz")
    np.savez_compressed(path, **out)
    print(f"wrote {path} ({os.path.getsize(path) / 1e6:.2f} MB)")


def init_guess_fixtures():
    """The reference's initial-guess pipeline around the NCC kernel: block_downsample, phase_correlation_shift,
    universal_median_test, fill_nan_grid, auto_pyramid_levels and pyramid_search (numba backend)."""
    from al_dvc.utils.inpaint import fill_nan_grid
    from al_dvc.utils.outlier_detection import universal_median_test

    out = {}
    rng = np.random.default_rng(31)
    v = rng.normal(0.0, 2.0, (20, 22, 26)).astype(np.float32)
    out["bd_vol"] = v
    for fac in (2, 3, 4):
        out[f"bd_{fac}"] = ris.block_downsample(v, fac)

    # phase correlation: a bead pair under a translation, at max_dim 128 (factor 1) and 24 (factor 4)
    pair = IG.raw_pc_pair()
    pf, pg = normalize_volume(pair.f), normalize_volume(pair.g)
    out.update(pc_sha_f=IG.sha(pf), pc_sha_g=IG.sha(pg), pc_shift=ris.phase_correlation_shift(pf, pg),
               pc_shift_md24=ris.phase_correlation_shift(pf, pg, None, 24))

    # median test and inpainting on a 7 x 8 x 9 vector field with outliers and holes
    gs = (7, 8, 9)
    zz, yy, xx = np.meshgrid(*(np.arange(n, dtype=np.float64) for n in gs), indexing="ij")
    field = np.stack([0.3 * xx + 0.1 * yy, -0.2 * zz + 0.05 * xx * yy / 8, 0.5 + 0.02 * zz * zz], -1)
    field += rng.normal(0.0, 0.02, field.shape)
    field[2, 3, 4] += (3.0, -2.0, 1.0)
    field[5, 1, 7] += (0.0, 4.0, 0.0)
    field[0, 0, 0] += (-2.5, 0.0, 0.0)
    valid = rng.random(gs) > 0.15
    out.update(mt_field=field, mt_valid=valid, mt_flag=universal_median_test(field, valid, 2.0))
    holes = field[..., 0].copy()
    holes[~valid] = np.nan
    out.update(fill_in=holes, fill_out=fill_nan_grid(holes))

    # pyramid search: 96^3 pair, translation plus a small shear, nodes every 10 voxels, 16^3 template, +-12
    pair = IG.raw_py_pair()
    yf, yg = normalize_volume(pair.f), normalize_volume(pair.g)
    x0, y0, z0 = ref_grid_axes(dvcpara_default().voi, IG.PY_SHAPE, (20, 20, 20), (10, 10, 10))
    pm = mesh_setup(x0, y0, z0)
    coords = np.round(pm.coordinates).astype(np.int64)
    shift = ris.phase_correlation_shift(yf, yg)
    levels = ris.auto_pyramid_levels(IG.PY_SHAPE, IG.PY_SUBSET, IG.PY_RADIUS, f=yf)
    info = ris.pyramid_search(yf, yg, coords, pm.grid_shape, IG.PY_SUBSET, IG.PY_RADIUS, 0, global_shift=shift, backend="numba")
    out.update(py_sha_f=IG.sha(yf), py_sha_g=IG.sha(yg), py_coords=coords, py_grid=np.array(pm.grid_shape), py_shift=shift,
               py_levels=levels, py_disp=info["disp"], py_ok=info["ok"], py_cc=info["cc"], py_pce=info["pce"],
               py_clipped=info["clipped"], py_expansions=info["expansions"],
               py_level_nok=np.array([d["n_ok"] for d in info["per_level"]]),
               py_level_radius=np.array([d["radius"] for d in info["per_level"]]),
               py_level_subset=np.array([d["subset"] for d in info["per_level"]]))
    path = os.path.join(HERE, "golden_init_guess.npz")
    np.savez_compressed(path, **out)
    print(f"wrote {path} ({os.path.getsize(path) / 1e6:.2f} MB); pyramid levels {levels}, shift {shift}")


def strain_fixtures():
    """The reference's strain module (strain/compute_strain.py, gradient_methods.py, strain_types.py) on a smooth
    nonlinear displacement over a 9 x 10 x 11 node grid with invalid nodes."""
    from al_dvc.strain.compute_strain import compute_strain
    from al_dvc.strain.gradient_methods import gradient_fd, gradient_plane_fit

    rng = np.random.default_rng(41)
    x0, y0, z0 = np.arange(11) * 6.0 + 10, np.arange(10) * 5.0 + 10, np.arange(9) * 7.0 + 10
    sm = mesh_setup(x0, y0, z0)
    N = sm.n_nodes
    X, Y, Z = (sm.coordinates[:, k] for k in range(3))
    U = np.column_stack([0.02 * X + 0.004 * Y - 3e-4 * X * Z + 0.3 * np.sin(Y / 17.0),
                         -0.015 * Y + 0.01 * Z + 2e-4 * X * X,
                         0.03 * Z - 0.02 * X + 0.1 * np.cos(X / 23.0) * np.sin(Z / 31.0)])
    U += rng.normal(0.0, 1e-3, U.shape)
    valid = rng.random(N) > 0.1
    valid[[0, 57, 300]] = False
    F_direct = rng.normal(0.0, 0.02, (N, 3, 3))
    sm.node_valid = valid
    out = {"st_x0": x0, "st_y0": y0, "st_z0": z0, "st_U": U, "st_valid": valid, "st_F_direct": F_direct,
           "st_boundary": sm.boundary_nodes}
    grid = sm.grid_shape
    Ug = U.reshape(grid + (3,)).copy()
    for hw in ((1, 1, 1), (2, 1, 1)):
        F, c = gradient_plane_fit(Ug, sm.spacing, hw, valid.reshape(grid))
        out[f"pf_{hw[0]}{hw[1]}{hw[2]}_F"], out[f"pf_{hw[0]}{hw[1]}{hw[2]}_complete"] = F, c
    F, c = gradient_fd(Ug, sm.spacing, valid.reshape(grid))
    out["fd_F"], out["fd_complete"] = F, c
    keys = ("disp_u", "disp_v", "disp_w", "F", "exx", "eyy", "ezz", "exy", "exz", "eyz", "principal", "max_shear",
            "von_mises", "volumetric", "det_F", "rotation_deg", "strain_valid")
    cases = {
        "inf_pf": dict(strain_type="infinitesimal", strain_method="plane_fit"),
        "gl_fd": dict(strain_type="green_lagrange", strain_method="fd"),
        "ea_pf2": dict(strain_type="euler_almansi", strain_method="plane_fit", strain_plane_fit_halfwidth=(2, 1, 1)),
        "he_direct": dict(strain_type="hencky", strain_method="direct", voxel_size=(0.5, 0.7, 1.3)),
        "inf_smooth": dict(strain_type="infinitesimal", strain_method="plane_fit", disp_smoothing=0.8, strain_smoothing=1.1,
                           strain_edge_trim=False),
    }
    for name, kw in cases.items():
        para = dvcpara_default(**kw)
        r = compute_strain(sm, para, U, F_direct=F_direct)
        for k in keys:
            out[f"cs_{name}_{k}"] = np.asarray(getattr(r, k))
    path = os.path.join(HERE, "golden_strain.npz")
    np.savez_compressed(path, **out)
    print(f"wrote {path} ({os.path.getsize(path) / 1e6:.2f} MB)")


def beta_fixtures():
    """The reference's beta auto-tune (solver/beta_tuning.py) on a 6 x 5 x 4 hex mesh with three invalid nodes, a
    smooth field plus noise, boundary nodes excluded, both scoring criteria."""
    from al_dvc.solver.beta_tuning import auto_tune_beta

    gm = mesh_setup(np.arange(6) * 6.0, np.arange(5) * 7.0, np.arange(4) * 5.0)
    nn = gm.n_nodes
    node_valid = np.ones(nn, dtype=bool)
    node_valid[[7, 8, 33]] = False
    elems = gm.elements.copy()
    bad = ~node_valid[elems].all(axis=1)
    elems[bad, :] = -1
    gm.elements = elems
    gm.node_valid = node_valid
    ops = build_fem_operators(gm, 2)
    rng = np.random.default_rng(51)
    X, Y, Z = (gm.coordinates[:, k] for k in range(3))
    U1 = np.column_stack([0.02 * X - 0.01 * Y, 0.015 * Z + 0.3 * np.sin(X / 9.0), -0.01 * X + 0.02 * Z]) + rng.normal(0, 0.05, (nn, 3))
    F1 = np.tile(np.array([[0.02, -0.01, 0.0], [0.0, 0.0, 0.015], [-0.01, 0.0, 0.02]]), (nn, 1, 1)) + rng.normal(0, 0.01, (nn, 3, 3))
    exclude = np.zeros(nn, dtype=bool)
    exclude[gm.boundary_nodes] = True
    exclude[[20, 21]] = True
    out = {"bt_U1": U1, "bt_F1": F1, "bt_exclude": exclude, "bt_elem_active": ~bad, "bt_grid": np.array(gm.grid_shape),
           "bt_spacing": np.array(gm.spacing)}
    for crit in ("matlab", "normalized"):
        para = dvcpara_default(winstepsize=(6, 6, 6), beta_criterion=crit, global_solver="pcg", pcg_tol=1e-10)
        beta, info = auto_tune_beta(ops, para, 1e-3, U1, F1, exclude)
        for k in ("betas", "err1", "err2", "score", "k_best"):
            out[f"bt_{crit}_{k}"] = np.asarray(info[k])
        out[f"bt_{crit}_beta"] = beta
    path = os.path.join(HERE, "golden_beta.npz")
    np.savez_compressed(path, **out)
    print(f"wrote {path} ({os.path.getsize(path) / 1e6:.2f} MB): betas {out['bt_matlab_betas']}, k {out['bt_matlab_k_best']}, "
          f"{out['bt_normalized_k_best']}, beta {out['bt_normalized_beta']}")


def pass_fixtures():
    """Whole frame pairs through the reference's own run_aldvc (core/pipeline.py, numba backend, PCG global
    solver, FEM global step, fixed beta): per case the node validity, the initial guess, the local 12-DOF
    result after outlier filling, the final U / F / status / ZNCC after the ADMM loop and its step count."""
    from al_dvc.core.pipeline import run_aldvc
    from al_dvc.io.volume_ops import normalize_volume

    import pass_inputs as PI

    out = {}
    for name, c in PI.PASS_CASES.items():
        f, g, mask, _ = PI.pass_pair(name)
        para = dvcpara_default(**PI.PASS_COMMON, **c["para"], backend="numba", verbose=False)
        r = run_aldvc(para, [f, g], masks=None if mask is None else [mask, None], compute_strain=False)
        fr = r.result_disp[0]
        m = r.dvc_mesh
        infos = fr.admm.local_info
        out.update({f"{name}_sha_f": PI.sha(normalize_volume(f)), f"{name}_sha_g": PI.sha(normalize_volume(g)),
                    f"{name}_coords": np.round(m.coordinates).astype(np.int64), f"{name}_grid": np.array(m.grid_shape),
                    f"{name}_spacing": np.array(m.spacing), f"{name}_node_valid": m.node_valid, f"{name}_U0": fr.U0,
                    f"{name}_U_local": fr.U_local, f"{name}_F_local": fr.F_local, f"{name}_U": fr.U, f"{name}_F": fr.F,
                    f"{name}_status": fr.status, f"{name}_zncc": fr.zncc, f"{name}_steps": fr.admm.n_steps,
                    f"{name}_status_local": infos[0].status, f"{name}_n_iter_local": infos[0].n_iter,
                    f"{name}_n_iter": infos[-1].n_iter})
        print(f"pass {name}: grid {m.grid_shape}, {fr.admm.n_steps} ADMM steps, statuses {np.bincount(fr.status.astype(int))}")
    path = os.path.join(HERE, "golden_pass.npz")
    np.savez_compressed(path, **out)
    print(f"wrote {path} ({os.path.getsize(path) / 1e6:.2f} MB)")


def ncc_fft_fixtures():
    """The reference's ncc_search where it takes its FP32 FFT branch (integer_search.py:395, :418-443): a 17^3
    template at +-9 and +-16, an anisotropic template and radius, and the expansion from +-8 (direct) to +-16 and
    +-32 (FFT); plus _window_box_stats on one node's window."""
    from al_dvc.io.volume_ops import normalize_volume

    import pass_inputs as PI

    pair = PI.ncc_pair()
    f, g = normalize_volume(pair.f), normalize_volume(pair.g)
    coords = PI.ncc_coords()
    shift = PI.ncc_shift(coords)
    out = {"sha_f": PI.sha(f), "sha_g": PI.sha(g), "coords": coords, "shift": shift}
    for name, c in PI.NCC_SEARCHES.items():
        res = ris.ncc_search(f, g, coords, c["subset"], c["radius"], shift if c["shift"] else None, backend="numba")
        for k in ("disp", "cc", "pce", "clipped", "ok"):
            out[f"{name}_{k}"] = res[k]
    res = ris.ncc_search_expanding(f, g, coords, PI.NCC_EXPAND["subset"], PI.NCC_EXPAND["radius"], None, True, 3, backend="numba")
    for k in ("disp", "cc", "pce", "clipped", "ok"):
        out[f"expand_{k}"] = res[k]
    out["expand_expansions"] = res["expansions"]
    out["expand_radius"] = np.array(res["radius"])
    W = np.ascontiguousarray(g[10:40, 12:42, 14:44][None])  # one 30^3 window, boxes of (sz, sy, sx) = (13, 11, 9)
    s1 = np.empty((1, 18, 20, 22))
    s2 = np.empty((1, 18, 20, 22))
    ris._window_box_stats(W, 13, 11, 9, s1, s2)
    out.update(box_W_origin=np.array([10, 12, 14]), box_sum=s1, box_sq=s2)
    path = os.path.join(HERE, "golden_ncc_fft.npz")
    np.savez_compressed(path, **out)
    print(f"wrote {path} ({os.path.getsize(path) / 1e6:.2f} MB); expansions {res['expansions']}, radius {res['radius']}")


# geometries of the tile plans: (volume shape, winsize, winstepsize, search radius, extra DVCPara fields, edges, disp
# field scale (0: none), restricted-node stride (0: all nodes))
TILING_CASES = {
    "base": ((96, 112, 128), 16, 8, 8, {}, (96, 112, 128), 0.0, 0),
    "disp": ((96, 112, 128), 16, 8, 8, {}, (112,), 3.7, 0),
    "aniso": ((90, 120, 150), (20, 32, 24), (10, 12, 8), (10, 8, 6),
              {"prefilter_sigma": 1.0, "tile_strain_margin": 0.5, "tile_disp_margin": 5}, (100, 140), 2.2, 0),
    "nodes": ((96, 112, 128), 16, 8, 8, {}, (96,), 1.5, 7),
    "small": ((96, 112, 128), 16, 8, 8, {}, (24, 0), 0.0, 0),
}


def tiling_fixtures():
    """The reference's tile plans (solver/tiling.py tile_pad :141, plan_tiles :204) over grid meshes of several
    geometries: halos, fallbacks, and per tile the node block and the box (origin, shape, open faces)."""
    from al_dvc.solver.tiling import plan_tiles, tile_pad

    out = {}
    for name, (shape, ws, step, rad, extra, edges, dscale, stride) in TILING_CASES.items():
        para = dvcpara_default(winsize=ws, winstepsize=step, search_radius=rad, verbose=False, **extra)
        x0, y0, z0 = ref_grid_axes(para.voi, shape, para.winsize, para.winstepsize)
        mesh = mesh_setup(x0, y0, z0)
        coords = np.round(mesh.coordinates).astype(np.int64)
        half = tuple(int(w) // 2 for w in np.broadcast_to(np.asarray(para.winsize), (3,)))
        rng = np.random.default_rng(7)
        disp = None if dscale == 0 else dscale * rng.uniform(-1.0, 1.0, size=(len(coords), 3))
        if disp is not None:
            disp[::11] = np.nan  # non-finite rows are ignored by the halo
        nodes = None if stride == 0 else np.arange(3, len(coords), stride)
        out[f"{name}_grid"] = np.array(mesh.grid_shape)
        out[f"{name}_coords"] = coords
        out[f"{name}_ref_pad"] = np.array(tile_pad(para, half))
        out[f"{name}_def_pad"] = np.array(tile_pad(para, half, disp=disp, deformed=True))
        if disp is not None:
            out[f"{name}_disp"] = disp
        if nodes is not None:
            out[f"{name}_nodes"] = nodes
        for e in edges:
            plan = plan_tiles(mesh.grid_shape, coords, shape, para, half, disp=disp, nodes=nodes, edge=e)
            key = f"{name}_e{e}"
            out[f"{key}_count"] = np.array([len(n) for n, _ in plan], dtype=np.int64)
            out[f"{key}_nodes"] = np.concatenate([n for n, _ in plan]).astype(np.int64)
            out[f"{key}_origin"] = np.array([b.origin for _, b in plan], dtype=np.int64)
            out[f"{key}_shape"] = np.array([b.shape for _, b in plan], dtype=np.int64)
            out[f"{key}_faces"] = np.array([b.open_faces for _, b in plan], dtype=bool)
            out[f"{key}_fallback"] = np.array(bool(plan.fallback))
    out["cases"] = np.array(list(TILING_CASES))
    path = os.path.join(HERE, "golden_tiling.npz")
    np.savez_compressed(path, **out)
    print(f"wrote {path} ({os.path.getsize(path) / 1e6:.2f} MB)")


def series_fixtures():
    """The reference's run_aldvc over a three-frame series (core/pipeline.py:82-452; cumulative displacements
    :455-491): per case and frame the reference frame, initial guess, local result, final U / F / ZNCC / statuses,
    outlier flags, cumulative displacement and ADMM step count; plus its interp_grid_field (utils/grid_interp.py) on
    random node grids, both orders, points inside and outside the grid."""
    from al_dvc.core.pipeline import run_aldvc
    from al_dvc.utils.grid_interp import interp_grid_field

    import pass_inputs as PI

    vols = PI.series_frames()
    out = {"sha": np.array([PI.sha(v) for v in vols])}
    for name, c in PI.SERIES_CASES.items():
        common = {k: v for k, v in PI.PASS_COMMON.items() if k != "init_guess_method"}
        para = dvcpara_default(**common, **PI.SERIES_PARA, init_guess_method=c["init_guess_method"],
                               reference_mode=c["reference_mode"], cumulative_interp=c["cumulative_interp"], backend="numba",
                               verbose=False)
        r = run_aldvc(para, vols, compute_strain=False)
        out[f"{name}_coords"] = r.dvc_mesh.coordinates
        for k, fr in enumerate(r.result_disp):
            key = f"{name}_f{k + 1}"
            out.update({f"{key}_ref": np.array(fr.ref_frame), f"{key}_U0": fr.U0, f"{key}_U_local": fr.U_local, f"{key}_U": fr.U,
                        f"{key}_F": fr.F, f"{key}_zncc": fr.zncc, f"{key}_status": fr.status, f"{key}_outlier": fr.outlier,
                        f"{key}_U_accum": fr.U_accum, f"{key}_steps": np.array(fr.admm.n_steps), f"{key}_U_std": fr.U_std})
        print(f"series {name}: {len(r.result_disp)} frames, steps {[fr.admm.n_steps for fr in r.result_disp]}")
    rng = np.random.default_rng(5)
    for gi, shape in enumerate(((5, 6, 7), (1, 6, 9), (12, 4, 3), (2, 2, 2))):
        nz, ny, nx = shape
        x0, y0, z0 = 10.0 + 12 * np.arange(nx), 5.0 + 12 * np.arange(ny), 7.0 + 12 * np.arange(nz)
        field = rng.normal(size=shape)
        q = np.stack([rng.uniform(x0[0] - 30, x0[-1] + 30, 300), rng.uniform(y0[0] - 30, y0[-1] + 30, 300),
                      rng.uniform(z0[0] - 30, z0[-1] + 30, 300)], 1)
        out.update({f"gi{gi}_field": field, f"gi{gi}_x0": x0, f"gi{gi}_y0": y0, f"gi{gi}_z0": z0, f"gi{gi}_q": q,
                    f"gi{gi}_o1": interp_grid_field(field, (x0, y0, z0), q, order=1),
                    f"gi{gi}_o3": interp_grid_field(field, (x0, y0, z0), q, order=3)})
    path = os.path.join(HERE, "golden_series.npz")
    np.savez_compressed(path, **out)
    print(f"wrote {path} ({os.path.getsize(path) / 1e6:.2f} MB)")


if __name__ == "__main__":
    which = sys.argv[1:] or ["kernels", "volume_ops", "init_guess", "strain", "beta", "pass", "ncc_fft", "tiling", "series"]
    makers = {"kernels": main, "volume_ops": volume_ops_fixtures, "init_guess": init_guess_fixtures, "strain": strain_fixtures,
              "beta": beta_fixtures, "pass": pass_fixtures, "ncc_fft": ncc_fft_fixtures, "tiling": tiling_fixtures,
              "series": series_fixtures}
    for w in which:
        makers[w]()
