"""GPU: the overlapping-quad copy of the deformed volume (``aldvc_make_quads``) and the IC-GN kernels reading their
cubic tap rows from it.  The copy must equal g[i..i+3] (clamped at the volume's last voxel) and the 12-DOF / 3-DOF
results with the copy must be bit-identical to those without it (the sampler forms the same products and sums in
the same order; NaN scores of invalid nodes compare equal), for Keys cubic and B-spline sampling, one subset shape
and per-node shapes with a mask.  Nodes that move into a NaN region of g while iterating (the lean kernel's
reference-frame sums are then swept again) match the oracle.
"""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

F_TRUE = np.array([[0.008, -0.003, 0.0], [0.002, -0.006, 0.004], [0.0, 0.003, 0.01]])
T_TRUE = np.array([-0.6, 0.9, 0.35])


def test_quads_equal_shifted_voxels():
    import torch

    from pyaldvc_b200 import kernels as K

    v = torch.from_numpy(np.random.default_rng(3).standard_normal(7 * 11 * 13).astype(np.float32)).cuda()
    q = K.make_quads(v).cpu().numpy()
    a = v.cpu().numpy()
    idx = np.minimum(np.arange(len(a))[:, None] + np.arange(4)[None, :], len(a) - 1)
    np.testing.assert_array_equal(q, a[idx])


@pytest.fixture(scope="module")
def pair(oracle_mod):
    from pyaldvc_b200 import synthetic as S

    shape = (56, 60, 64)
    c, pk = S.draw_beads(shape, 0.03, 21)
    centre = (32.0, 30.0, 28.0)
    f = S.normalize_volume(S.render_beads(shape, c, pk, 1.5))
    g = S.normalize_volume(S.render_beads(shape, S.displace_beads(c, S.affine(F_TRUE, T_TRUE, centre)), pk, 1.5))
    gx, gy, gz = oracle_mod.compute_gradients(f)
    zz, yy, xx = np.meshgrid(*(np.arange(n) for n in shape), indexing="ij")
    mask = (((xx - 32.0) ** 2 + (yy - 30.0) ** 2 + (zz - 28.0) ** 2) <= 22.0**2).astype(np.uint8)
    Z, Y, X = np.meshgrid(np.arange(14, 43, 7), np.arange(14, 47, 8), np.arange(14, 51, 9), indexing="ij")
    coords = np.stack([X.ravel(), Y.ravel(), Z.ravel()], 1).astype(np.int64)
    rng = np.random.default_rng(5)
    P0 = np.zeros((len(coords), 12))
    P0[:, 9:] = T_TRUE + (coords - np.array(centre)) @ F_TRUE.T + rng.uniform(-0.4, 0.4, size=(len(coords), 3))
    node_half = np.array([(6, 6, 8), (8, 8, 8), (7, 6, 7)], np.int32)[rng.integers(0, 3, size=len(coords))]
    return f, g, gx, gy, gz, mask, coords, P0, node_half


@pytest.mark.parametrize("mode", [1, 2], ids=["cubic", "bspline"])
@pytest.mark.parametrize("uneven", [False, True], ids=["one_shape", "per_node_masked"])
def test_icgn_with_quads_is_bit_identical(pair, mode, uneven):
    import torch

    from pyaldvc_b200 import kernels as K

    f, g, gx, gy, gz, mask, coords, P0, node_half = pair
    d = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    fd, gd, gxd, gyd, gzd, cd = (d(a) for a in (f, g, gx, gy, gz, coords))
    md, nhd = (d(mask), d(node_half)) if uneven else (None, None)
    half = tuple(int(v) for v in node_half.max(axis=0)) if uneven else (8, 8, 8)
    H, L, mf, bf, nv, valid = K.precompute(cd, half, fd, gxd, gyd, gzd, md, 0.5, 1e12, 1, None, None, nhd)
    assert int(valid.sum()) > 60
    g4 = K.make_quads(gd)
    for threads in (32, 128):
        kw = dict(variant=K.BATCHED, threads=threads, brick_floats=0, node_half=nhd)
        a = K.icgn12(cd, d(P0), half, fd, gxd, gyd, gzd, md, gd, mode, L, mf, valid, 1e-2, 1e-3, 100, 5, **kw)
        b = K.icgn12(cd, d(P0), half, fd, gxd, gyd, gzd, md, gd, mode, L, mf, valid, 1e-2, 1e-3, 100, 5, g4=g4, **kw)
        for x, y, name in zip(a, b, ("P", "n_iter", "status", "zncc")):
            np.testing.assert_array_equal(x.cpu().numpy(), y.cpu().numpy(), err_msg=f"icgn12 {name} (threads {threads})")
        if mode == 1:
            assert float((a[2][valid.bool()] == 0).float().mean()) > 0.9
        P = a[0]
        U_old, F_fixed, vdual = P[:, 9:].contiguous(), P[:, :9].contiguous(), torch.zeros_like(P[:, 9:])
        a3 = K.icgn3(cd, U_old, F_fixed, vdual, half, fd, gxd, gyd, gzd, md, gd, mode, H, mf, bf, valid, 1e-3, 1e-2, 1e-3,
                     100, 5, **kw)
        b3 = K.icgn3(cd, U_old, F_fixed, vdual, half, fd, gxd, gyd, gzd, md, gd, mode, H, mf, bf, valid, 1e-3, 1e-2, 1e-3,
                     100, 5, g4=g4, **kw)
        for x, y, name in zip(a3, b3, ("U", "n_iter", "status", "zncc")):
            np.testing.assert_array_equal(x.cpu().numpy(), y.cpu().numpy(), err_msg=f"icgn3 {name} (threads {threads})")


@pytest.mark.parametrize("ndof", [12, 3])
def test_lean_kernel_nodes_reaching_nan_samples_match_oracle(oracle_mod, ndof):
    """Deformed-frame NaN (a masked slab of g, x >= 40): nodes whose subset is clear of it at P0 move into its
    cubic footprint while iterating.  The lean kernel takes the reference-frame sums of a node from its first
    complete sweep; an iteration that meets a NaN sample must sweep every sum again (the oracle leaves such voxels
    out of all the sums).  Same parity bar as test_gpu_parity.py."""
    import torch

    from pyaldvc_b200 import kernels as K
    from pyaldvc_b200 import synthetic as S
    from test_gpu_parity import assert_parity

    shape = (64, 64, 64)
    c, pk = S.draw_beads(shape, 0.03, 33)
    T = np.array([1.2, -0.3, 0.2])
    f = S.normalize_volume(S.render_beads(shape, c, pk, 1.5))
    g = S.normalize_volume(S.render_beads(shape, S.displace_beads(c, S.translation(T)), pk, 1.5))
    g[:, :, 40:] = np.nan
    gx, gy, gz = oracle_mod.compute_gradients(f)
    Z, Y, X = np.meshgrid(np.arange(12, 52, 5), np.arange(12, 52, 5), np.array([30, 31, 32]), indexing="ij")
    coords = np.stack([X.ravel(), Y.ravel(), Z.ravel()], 1).astype(np.int64)
    rng = np.random.default_rng(8)
    P0 = np.zeros((len(coords), 12))
    P0[:, 9:] = T + rng.uniform(-0.4, 0.4, size=(len(coords), 3))
    h = 6
    ones = np.ones((1, 1, 1), np.uint8)
    H, L, mf, bf, nv, valid = oracle_mod.precompute_nodes(coords, h, h, h, f, gx, gy, gz, ones, 0.5, 1e12)
    d = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    fd, gd, gxd, gyd, gzd, cd = (d(a) for a in (f, g, gx, gy, gz, coords))
    Hd, Ld, mfd, bfd, vd = d(H), d(L), d(mf), d(bf), d(valid.astype(np.uint8))
    if ndof == 12:
        ref = oracle_mod.icgn_12dof_parallel(coords, P0, h, h, h, f, gx, gy, gz, ones, g, 1, L, mf, bf, valid, 1e-3, 1e-4,
                                             100, 5)
        got = K.icgn12(cd, d(P0), (h, h, h), fd, gxd, gyd, gzd, None, gd, 1, Ld, mfd, vd, 1e-3, 1e-4, 100, 5,
                       variant=K.BATCHED, threads=128, brick_floats=0, g4=K.make_quads(gd))
        x_end = ref[0][:, 9]
    else:
        U_old, F_fixed, vdual = P0[:, 9:].copy(), np.zeros((len(coords), 3, 3)), np.zeros((len(coords), 3))
        ref = oracle_mod.icgn_3dof_parallel(coords, U_old, F_fixed, vdual, h, h, h, f, gx, gy, gz, ones, g, 1, H, mf, bf,
                                            valid, 1e-3, 1e-3, 1e-4, 100, 5)
        got = K.icgn3(cd, d(U_old), d(F_fixed), d(vdual), (h, h, h), fd, gxd, gyd, gzd, None, gd, 1, Hd, mfd, bfd, vd, 1e-3,
                      1e-3, 1e-4, 100, 5, variant=K.BATCHED, threads=128, brick_floats=0, g4=K.make_quads(gd))
        x_end = ref[0][:, 0]
    # the subset's last column samples taps up to floor(x) + 2: NaN once x >= 38
    far = coords[:, 0] + h
    clear_at_start = far + P0[:, 9] < 38.0
    crossing = clear_at_start & (far + x_end >= 38.0) & (ref[2] == 0)
    assert crossing.sum() >= 5, "too few nodes move into the NaN footprint"
    assert_parity(tuple(ref), tuple(t.cpu().numpy() for t in got), what=f"icgn{ndof} NaN slab")
