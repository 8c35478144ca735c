"""CPU: the tiled pass's geometry (pyaldvc_b200.tiling) against the reference's planner.

golden_tiling.npz holds the reference's own tile_pad and plan_tiles (solver/tiling.py:141-289) on five geometries
(made by tests/golden/make_golden.py tiling): cubic and anisotropic subsets, a measured displacement field with
non-finite rows, presmoothing and both halo margins, a restricted node set (the escape retry) and targets below
one subset (the whole-volume fallback) or at 0 (off).  The planner here must give the same halos, node blocks and
boxes.  The integer-search boxes, which the reference does not tile, are checked by construction: every node's
template and clamped search window inside its box, and the box's own clamp equal to the volume's.
"""

from __future__ import annotations

import os

import numpy as np
import pytest

from pyaldvc_b200 import tiling as T
from pyaldvc_b200.mesh import build_grid_axes, grid_coords
from pyaldvc_b200.pipeline import PassParams

HERE = os.path.dirname(os.path.abspath(__file__))

# the geometries of make_golden.TILING_CASES: (volume shape, winsize, winstepsize, search radius, extra fields, edges)
CASES = {
    "base": ((96, 112, 128), 16, 8, 8, {}, (96, 112, 128)),
    "disp": ((96, 112, 128), 16, 8, 8, {}, (112,)),
    "aniso": ((90, 120, 150), (20, 32, 24), (10, 12, 8), (10, 8, 6),
              {"prefilter_sigma": 1.0, "tile_strain_margin": 0.5, "tile_disp_margin": 5}, (100, 140)),
    "nodes": ((96, 112, 128), 16, 8, 8, {}, (96,)),
    "small": ((96, 112, 128), 16, 8, 8, {}, (24, 0)),
}


def _t3(v):
    return tuple(int(x) for x in np.broadcast_to(np.asarray(v), (3,)))


@pytest.fixture(scope="module")
def gt():
    with np.load(os.path.join(HERE, "golden", "golden_tiling.npz")) as z:
        return {k: z[k] for k in z.files}


def _case(name):
    shape, ws, step, rad, extra, edges = CASES[name]
    p = PassParams(winsize=_t3(ws), winstepsize=_t3(step), search_radius=_t3(rad), **extra)
    x0, y0, z0 = build_grid_axes(shape, p.winsize, p.winstepsize)
    coords = np.round(grid_coords(x0, y0, z0)).astype(np.int64)
    return shape, p, (len(z0), len(y0), len(x0)), coords, tuple(w // 2 for w in p.winsize), edges


@pytest.mark.parametrize("name", list(CASES))
def test_halos_and_plans_match_the_reference_planner(gt, name):
    shape, p, grid, coords, half, edges = _case(name)
    np.testing.assert_array_equal(grid, gt[f"{name}_grid"])
    np.testing.assert_array_equal(coords, gt[f"{name}_coords"])
    disp = gt.get(f"{name}_disp")
    nodes = gt.get(f"{name}_nodes")
    assert T.tile_pad(p, half) == tuple(gt[f"{name}_ref_pad"])
    assert T.tile_pad(p, half, disp=disp, deformed=True) == tuple(gt[f"{name}_def_pad"])
    for e in edges:
        key = f"{name}_e{e}"
        plan = T.plan_tiles(grid, coords, shape, p, half, disp=disp, nodes=nodes, edge=e)
        assert bool(plan.fallback) == bool(gt[f"{key}_fallback"])
        np.testing.assert_array_equal([len(t.nodes) for t in plan], gt[f"{key}_count"], err_msg=key)
        np.testing.assert_array_equal(np.concatenate([t.nodes for t in plan]), gt[f"{key}_nodes"], err_msg=key)
        np.testing.assert_array_equal([t.box.origin for t in plan], gt[f"{key}_origin"], err_msg=key)
        np.testing.assert_array_equal([t.box.shape for t in plan], gt[f"{key}_shape"], err_msg=key)
        np.testing.assert_array_equal([t.box.open_faces for t in plan], gt[f"{key}_faces"], err_msg=key)


def test_plan_covers_every_node_once_and_holds_its_windows():
    shape, p, grid, coords, half, _ = _case("base")
    plan = T.plan_tiles(grid, coords, shape, p, half, edge=96)
    assert len(plan) > 1 and not plan.fallback
    np.testing.assert_array_equal(np.sort(np.concatenate([t.nodes for t in plan])), np.arange(len(coords)))
    pad = tuple(max(a, b) for a, b in zip(plan.ref_pad, plan.def_pad))
    for t in plan:
        assert t.box.contains_windows(coords[t.nodes], plan.ref_pad)
        assert all(o >= 0 for o in t.box.origin) and all(o + n <= s for o, n, s in zip(t.box.origin, t.box.shape, shape))
        # a whole sub-lattice block carries its axes, in the C order of its nodes
        iz, iy, ix = t.axes
        lattice = (iz[:, None, None] * grid[1] + iy[None, :, None]) * grid[2] + ix[None, None, :]
        np.testing.assert_array_equal(t.nodes, lattice.ravel())
        # a face is open exactly where the halo did not reach the volume's face
        c = coords[t.nodes]
        for k_zyx, k_xyz in ((0, 2), (1, 1), (2, 0)):
            lo_want = int(c[:, k_xyz].min()) - pad[k_xyz]
            hi_want = int(c[:, k_xyz].max()) + pad[k_xyz] + 1
            assert t.box.open_faces[2 * k_zyx] == (lo_want > 0)
            assert t.box.open_faces[2 * k_zyx + 1] == (hi_want < shape[k_zyx])


def test_restricted_plan_and_quantised_pad():
    shape, p, grid, coords, half, _ = _case("base")
    nodes = np.array([5, 77, 300, 301, len(coords) - 1])
    pad = T._quantised((17, 20, 31))
    assert pad == (24, 24, 32)
    plan = T.plan_tiles(grid, coords, shape, p, half, nodes=nodes, edge=96, pad=pad)
    np.testing.assert_array_equal(np.sort(np.concatenate([t.nodes for t in plan])), nodes)
    for t in plan:
        # the box holds the given halo, except where the volume's own faces cut it
        c = coords[t.nodes]
        for k_zyx, k_xyz in ((0, 2), (1, 1), (2, 0)):
            assert t.box.origin[k_zyx] == max(0, int(c[:, k_xyz].min()) - pad[k_xyz])
            assert t.box.origin[k_zyx] + t.box.shape[k_zyx] == min(shape[k_zyx], int(c[:, k_xyz].max()) + pad[k_xyz] + 1)
        # a block with nodes left out carries no lattice axes (the grid-form precompute needs a whole sub-lattice)
        assert t.axes is None or len(t.nodes) == np.prod([len(a) for a in t.axes])


def test_box_crop_shift_and_growth():
    vol = np.arange(np.prod((40, 50, 60)), dtype=np.float32).reshape(40, 50, 60)
    box = T.Box((4, 8, 12), (20, 24, 28), (True, True, True, True, True, False))
    crop = box.crop(vol)
    assert crop.shape == (20, 24, 28) and crop.flags.c_contiguous
    c = np.array([[20, 15, 10], [30, 20, 12]])
    for (x, y, z), (xs, ys, zs) in zip(c, box.shift(c)):
        assert crop[zs, ys, xs] == vol[z, y, x]
    big, inner = box.grown((6, 9, 40), vol.shape)
    assert big.origin == (0, 0, 0) and big.shape == (30, 41, 60)
    np.testing.assert_array_equal(big.crop(vol)[inner], crop)
    whole = T.whole_box(vol.shape)
    assert whole.is_whole and whole.crop(vol) is vol
    b = T.box_for_ranges((-3, 10, 0), (40, 60, 59), vol.shape)
    assert b.origin == (0, 10, 0) and b.shape == (40, 40, 59) and b.open_faces == (False, False, True, False, False, True)


def test_slab_ranges_cover_the_volume_in_whole_blocks():
    for shape, voxels, step in (((37, 20, 30), 600 * 7, 1), ((37, 20, 30), 600 * 7, 4), ((10, 8, 8), 1, 3), ((64, 4, 4), 1 << 30, 8)):
        sl = T.slab_ranges(shape, voxels, step)
        assert sl[0][0] == 0 and sl[-1][1] == shape[0]
        assert all(a[1] == b[0] for a, b in zip(sl, sl[1:]))
        assert all((z1 - z0) % step == 0 for z0, z1 in sl[:-1])
        assert all((z1 - z0) * shape[1] * shape[2] <= max(voxels, step * shape[1] * shape[2]) for z0, z1 in sl)


@pytest.mark.parametrize("edge", [0, 60, 90])
@pytest.mark.parametrize("shifted", [False, True])
def test_ncc_boxes_hold_every_read_and_clamp_like_the_volume(edge, shifted):
    shape = (70, 90, 110)
    half, radius = (8, 6, 7), (9, 8, 10)
    x0, y0, z0 = build_grid_axes(shape, (16, 12, 14), (10, 9, 11))
    coords = np.round(grid_coords(x0, y0, z0)).astype(np.int64)
    rng = np.random.default_rng(3)
    shift = rng.integers(-20, 21, size=coords.shape) if shifted else None
    groups = T.plan_ncc_boxes(coords, half, radius, shift, shape, edge)
    np.testing.assert_array_equal(np.sort(np.concatenate([g for g, _ in groups])), np.arange(len(coords)))
    if edge == 0:
        assert len(groups) == 1
    else:
        assert len(groups) > 1
    sh = np.zeros_like(coords) if shift is None else shift
    for sel, box in groups:
        o_xyz = np.array(box.origin[::-1])
        n_xyz = np.array(box.shape[::-1])
        for k in range(3):
            h, r, n = half[k], radius[k], shape[2 - k]
            W = 2 * h + 1 + 2 * r
            c, s = coords[sel, k], sh[sel, k]
            w_vol = np.clip(c + s - h - r, 0, n - W)  # the search's clamp in the volume
            w_box = np.clip(c - o_xyz[k] + s - h - r, 0, n_xyz[k] - W)  # and in the box
            np.testing.assert_array_equal(w_box + o_xyz[k], w_vol)
            assert (w_box >= 0).all() and (w_box + W <= n_xyz[k]).all()
            t_lo, t_hi = np.maximum(c - h, 0), np.minimum(c + h + 1, n)  # the template, where it is in the volume
            assert (t_lo >= o_xyz[k]).all() and (t_hi <= o_xyz[k] + n_xyz[k]).all()
            # a template cut by the volume is cut by the box at the same face
            assert ((c - h < 0) <= (o_xyz[k] == 0)).all() and ((c + h + 1 > n) <= (o_xyz[k] + n_xyz[k] == n)).all()


def test_nodes_leaving_an_open_face_are_retried_with_a_wider_halo(monkeypatch):
    """The escape retry (local_icgn.py:448-459): a fake solve marks a node out of bounds when its box does not
    hold the 30 voxels its subset needs (clipped by the volume); the plan is repeated for those nodes with the halo
    widened until it does."""
    import torch

    shape, p, grid, coords, half, _ = _case("base")
    need = 30
    status = torch.zeros(len(coords), dtype=torch.int8)
    rounds = []

    def plan_fn(nodes, pad):
        return T.plan_tiles(grid, coords, shape, p, half, nodes=nodes, edge=96, pad=pad)

    def solve(t):
        rounds.append(len(t.nodes))
        c = coords[t.nodes]
        ok = np.ones(len(t.nodes), dtype=bool)
        for k_zyx, k_xyz in ((0, 2), (1, 1), (2, 0)):
            lo = np.maximum(c[:, k_xyz] - need, 0)
            hi = np.minimum(c[:, k_xyz] + need, shape[k_zyx] - 1)
            ok &= (lo >= t.box.origin[k_zyx]) & (hi <= t.box.origin[k_zyx] + t.box.shape[k_zyx] - 1)
        status[torch.from_numpy(t.nodes)] = torch.from_numpy(np.where(ok, 0, T.STATUS_OUT_OF_BOUNDS).astype(np.int8))

    # the host logic alone: the tiles in turn on the host instead of alternating CUDA streams
    monkeypatch.setattr(T, "_on_streams", lambda items, fn: [fn(t) for t in items])
    rec = T.TileRecord()
    retried = T._solve_tiles(plan_fn, solve, status, "icgn", rec, (16, 16, 16), (8, 8, 8))
    assert retried > 0 and rec.stages["icgn_retry"]["calls"] == 2  # halos 24 (still short) and 32
    assert int((status != 0).sum()) == 0
    assert sum(rounds) == len(coords) + retried


def test_left_volume_decides_on_the_warped_corners():
    """A node's last iterate leaves the volume when a corner of its warped subset is outside the sampling margin
    [1, n - 3] (interp_kernels.interp_margin_ok) of the volume; shapes (nz, ny, nx) = (40, 50, 60)."""
    shape = (40, 50, 60)
    half, stride = (8, 6, 5), 1
    c = np.array([[30, 25, 20]] * 6)  # x, y, z
    P = np.zeros((6, 12))
    P[1, 9] = 60 - 3 - 38 + 0.5   # x corner 38 + u = 57.5 > 57
    P[2, 9] = 60 - 3 - 38 - 1e-6  # just inside
    P[3, 11] = -(28 - 1) - 0.25   # z corner 20 - 8 + w = -15.25 < 1
    P[4, 0] = 0.3                 # stretch: x corner 30 + 1.3 * 8 = 40.4, inside
    P[5, 8] = 0.9                 # z stretch alone keeps the corners inside: 20 -+ 1.9 * 8 = 4.8 .. 35.2
    P[5, 7] = 3.0                 # plus 3 Y: 20 + 1.9 * 8 + 3 * 6 = 53.2 > 37
    got = T.left_volume(P, c, half, stride, shape)
    np.testing.assert_array_equal(got, [False, True, False, True, False, True])
    # with a stride the last sample of an axis stops short of +h: 2h = 16, stride 3 -> offsets -8 .. +7
    P2 = np.zeros((1, 12))
    P2[0, 9] = 60 - 3 - 37 - 0.5  # corner at 30 + 7 + u = 56.5: inside with stride 3, outside the +8 corner
    assert not T.left_volume(P2, c[:1], half, 3, shape)[0]
    assert T.left_volume(P2, c[:1], half, 1, shape)[0]
