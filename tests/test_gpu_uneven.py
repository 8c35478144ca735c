"""Uneven batch: nodes with different anisotropic subset shapes and a reference mask, in ONE persistent
precompute / 12-DOF / 3-DOF launch each, against the FP64 oracle called once per subset shape (the reference
calls its kernels once per shape).  Same parity bar as test_gpu_parity.py.

Inputs: a seeded bead pair under an affine deformation, a spherical reference mask (so the masked voxel count
varies per node), a 6^3 node grid with five subset shapes from 13 x 13 x 19 to 19^3.
"""

from __future__ import annotations

import numpy as np
import pytest

from test_gpu_parity import assert_parity

pytestmark = pytest.mark.gpu

SHAPES = np.array([(6, 6, 9), (8, 8, 8), (7, 7, 10), (9, 9, 9), (6, 8, 7)], dtype=np.int32)
F_TRUE = np.array([[0.01, 0.004, 0.0], [-0.003, -0.008, 0.002], [0.0, 0.005, 0.012]])
T_TRUE = np.array([0.7, -1.1, 0.45])


@pytest.fixture(scope="module")
def problem(oracle_mod):
    from pyaldvc_b200 import synthetic as S

    shape = (72, 72, 72)
    c, pk = S.draw_beads(shape, 0.03, 9)
    centre = (36.0, 36.0, 36.0)
    f = S.normalize_volume(S.render_beads(shape, c, pk, 1.5))
    g = S.normalize_volume(S.render_beads(shape, S.displace_beads(c, S.affine(F_TRUE, T_TRUE, centre)), pk, 1.5))
    gx, gy, gz = oracle_mod.compute_gradients(f)
    zz, yy, xx = np.meshgrid(*(np.arange(72),) * 3, indexing="ij")
    mask = (((xx - 36.0) ** 2 + (yy - 36.0) ** 2 + (zz - 36.0) ** 2) <= 27.0**2).astype(np.uint8)
    ax = np.arange(16, 57, 8)
    gz_, gy_, gx_ = np.meshgrid(ax, ax, ax, indexing="ij")
    coords = np.stack([gx_.ravel(), gy_.ravel(), gz_.ravel()], 1).astype(np.int64)
    rng = np.random.default_rng(12)
    node_half = SHAPES[rng.integers(0, len(SHAPES), size=len(coords))]
    X = coords - np.array(centre)
    U = T_TRUE + X @ F_TRUE.T
    P0 = np.zeros((len(coords), 12))
    P0[:, 9:] = U + rng.uniform(-0.4, 0.4, size=U.shape)
    return f, g, gx, gy, gz, mask, coords, node_half, P0


def _oracle_by_shape(oracle_mod, prob, fn):
    """Run ``fn(sel, hx, hy, hz)`` per subset shape and scatter its outputs back into node order."""
    *_, coords, node_half, _ = prob
    outs = None
    for sh in np.unique(node_half, axis=0):
        sel = np.flatnonzero((node_half == sh).all(axis=1))
        res = fn(sel, *(int(v) for v in sh))
        if outs is None:
            outs = [np.zeros((len(coords),) + np.asarray(r).shape[1:], dtype=np.asarray(r).dtype) for r in res]
        for o, r in zip(outs, res):
            o[sel] = r
    return outs


@pytest.mark.parametrize("variant", [0, 1], ids=["batched", "plain"])
def test_uneven_masked_batch_matches_oracle_per_shape(oracle_mod, problem, variant):
    import torch

    from pyaldvc_b200 import kernels as K

    f, g, gx, gy, gz, mask, coords, node_half, P0 = problem
    hmax = tuple(int(v) for v in node_half.max(axis=0))
    d = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    fd, gd, gxd, gyd, gzd, md, cd, nhd = (d(a) for a in (f, g, gx, gy, gz, mask, coords, node_half))

    # precompute
    pre_o = _oracle_by_shape(oracle_mod, problem, lambda s, hx, hy, hz: oracle_mod.precompute_nodes(
        coords[s], hx, hy, hz, f, gx, gy, gz, mask, 0.5, 1e12))
    H, L, mf, bf, nv, valid = K.precompute(cd, hmax, fd, gxd, gyd, gzd, md, 0.5, 1e12, 1, None, None, nhd)
    np.testing.assert_array_equal(valid.cpu().numpy().astype(bool), pre_o[5])
    np.testing.assert_array_equal(nv.cpu().numpy(), pre_o[4])
    ok = pre_o[5]
    assert ok.sum() > 100 and len(np.unique(pre_o[4][ok])) > 20  # masked counts vary per node
    Hr = pre_o[0]
    np.testing.assert_allclose(H.cpu().numpy()[ok], Hr[ok], rtol=1e-4, atol=1e-5 * np.abs(Hr[ok]).max())

    # 12-DOF, one launch for every shape
    ref12 = _oracle_by_shape(oracle_mod, problem, lambda s, hx, hy, hz: oracle_mod.icgn_12dof_parallel(
        coords[s], P0[s], hx, hy, hz, f, gx, gy, gz, mask, g, 1, pre_o[1][s], pre_o[2][s], pre_o[3][s], pre_o[5][s], 1e-2,
        1e-3, 100, 5))
    got12 = K.icgn12(cd, d(P0), hmax, fd, gxd, gyd, gzd, md, gd, 1, L, mf, valid, 1e-2, 1e-3, 100, 5, variant=variant,
                     node_half=nhd)
    got12 = tuple(t.cpu().numpy() for t in got12)
    assert_parity(tuple(ref12), got12, what="uneven icgn12")
    assert np.mean(ref12[2][ok] == 0) > 0.9

    # 3-DOF (ADMM subproblem 1) from the 12-DOF result
    P = ref12[0]
    U_old, F_fixed = P[:, 9:].copy(), P[:, :9].reshape(-1, 3, 3).copy()
    vdual = np.zeros_like(U_old)
    ref3 = _oracle_by_shape(oracle_mod, problem, lambda s, hx, hy, hz: oracle_mod.icgn_3dof_parallel(
        coords[s], U_old[s], F_fixed[s], vdual[s], hx, hy, hz, f, gx, gy, gz, mask, g, 1, pre_o[0][s], pre_o[2][s], pre_o[3][s],
        pre_o[5][s], 1e-3, 1e-2, 1e-3, 100, 5))
    got3 = K.icgn3(cd, d(U_old), d(F_fixed), d(vdual), hmax, fd, gxd, gyd, gzd, md, gd, 1, H, mf, bf, valid, 1e-3, 1e-2, 1e-3, 100,
                   5, variant=variant, node_half=nhd)
    got3 = tuple(t.cpu().numpy() for t in got3)
    assert_parity(tuple(ref3), got3, what="uneven icgn3")


def test_node_shape_beyond_the_call_maximum_is_invalid(problem):
    import torch

    from pyaldvc_b200 import kernels as K
    from pyaldvc_b200.cuda_kernels import STATUS_INVALID_SUBSET as STATUS_INVALID

    f, g, gx, gy, gz, mask, coords, node_half, P0 = problem
    d = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    nh = node_half[:8].copy()
    nh[3] = (9, 9, 12)  # above the maximum passed below
    hmax = (9, 9, 10)
    fd, gd, gxd, gyd, gzd = (d(a) for a in (f, g, gx, gy, gz))
    H, L, mf, bf, nv, valid = K.precompute(d(coords[:8]), hmax, fd, gxd, gyd, gzd, None, 0.5, 1e12, 1, None, None, d(nh))
    assert valid.cpu().numpy()[3] == 0
    ones = torch.ones(8, dtype=torch.uint8, device="cuda")  # force the node in: the solver must still refuse it
    _, _, st, _ = K.icgn12(d(coords[:8]), d(P0[:8]), hmax, fd, gxd, gyd, gzd, None, gd, 1, L, mf, ones, 1e-2, 1e-3, 100, 5,
                           node_half=d(nh))
    assert st.cpu().numpy()[3] == STATUS_INVALID
