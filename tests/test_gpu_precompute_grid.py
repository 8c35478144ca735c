"""GPU: the separable precompute on a tensor node grid (``aldvc_precompute_grid``) against the reference's outputs
(golden fixtures: the stride-1 cases with stored gradients, masked and unmasked) and against the per-node kernel and
the FP64 oracle on a bead volume whose grid has nodes past the volume edges, with and without a spherical mask.  Same bar as the per-node kernel (test_gpu_parity.py): validity and
voxel counts identical, H within 1e-4 relative (1e-5 of its largest entry), meanf / bottomf within 1e-5.
"""

from __future__ import annotations

import numpy as np
import pytest

from test_oracle_golden import pre_args

pytestmark = pytest.mark.gpu


def _check(got, ref_H, ref_L, ref_mf, ref_bf, ref_nv, ref_valid, what):
    H, L, mf, bf, nv, valid = (t.cpu().numpy() for t in got)
    ok = ref_valid.astype(bool)
    np.testing.assert_array_equal(valid.astype(bool), ok, err_msg=f"{what}: valid")
    np.testing.assert_array_equal(nv, ref_nv, err_msg=f"{what}: n_valid")
    np.testing.assert_allclose(H[ok], ref_H[ok], rtol=1e-4, atol=1e-5 * np.abs(ref_H[ok]).max(), err_msg=f"{what}: H")
    np.testing.assert_allclose(mf[ok], ref_mf[ok], rtol=1e-5, atol=1e-6, err_msg=f"{what}: meanf")
    np.testing.assert_allclose(bf[ok], ref_bf[ok], rtol=1e-5, err_msg=f"{what}: bottomf")
    np.testing.assert_allclose(L[ok], ref_L[ok], rtol=1e-3, atol=1e-4 * np.abs(ref_L[ok]).max(), err_msg=f"{what}: L")


@pytest.mark.parametrize("name", ["plain", "aniso", "masked"])
def test_grid_precompute_matches_reference(golden, name):
    import torch

    from pyaldvc_b200 import kernels as K

    c, (gx, gy, gz), mask, _ = pre_args(golden, name)
    d = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    xs, ys, zs = (np.round(golden[k]).astype(np.int64) for k in ("x0", "y0", "z0"))
    m = d(mask) if c["mask"] else None
    got = K.precompute_grid(xs, ys, zs, c["h"], d(golden["f"]), d(gx), d(gy), d(gz), 0.5, 1e12, m)
    _check(got, *(golden[f"pre_{name}_{k}"] for k in ("H", "L", "meanf", "bottomf", "n_valid", "valid")), name)


@pytest.mark.parametrize("masked", [False, True], ids=["unmasked", "masked"])
def test_grid_precompute_matches_per_node_kernel_and_oracle(oracle_mod, masked):
    import torch

    from pyaldvc_b200 import kernels as K
    from pyaldvc_b200 import synthetic as S

    shape = (64, 64, 64)
    c, pk = S.draw_beads(shape, 0.03, 17)
    f = S.normalize_volume(S.render_beads(shape, c, pk, 1.5))
    gx, gy, gz = oracle_mod.compute_gradients(f)
    xs, ys, zs = np.array([5, 16, 30, 47, 60]), np.array([12, 30, 51]), np.array([9, 33, 55])  # 5 and 60: subsets outside
    Z, Y, X = np.meshgrid(zs, ys, xs, indexing="ij")
    coords = np.stack([X.ravel(), Y.ravel(), Z.ravel()], 1).astype(np.int64)
    d = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    half = (8, 8, 8)
    if masked:  # a sphere of radius 24: masked voxel counts vary per node, some nodes fall below half a subset
        zz, yy, xx = np.meshgrid(*(np.arange(64),) * 3, indexing="ij")
        mask = (((xx - 31.5) ** 2 + (yy - 31.5) ** 2 + (zz - 31.5) ** 2) <= 24.0**2).astype(np.uint8)
    else:
        mask = np.ones((1, 1, 1), np.uint8)
    md = d(mask) if masked else None
    got = K.precompute_grid(xs, ys, zs, half, d(f), d(gx), d(gy), d(gz), 0.5, 1e12, md)
    ref = oracle_mod.precompute_nodes(coords, *half, f, gx, gy, gz, mask, 0.5, 1e12)
    assert ref[5].sum() > 5 and (~ref[5].astype(bool)).sum() > 10
    if masked:
        assert len(np.unique(ref[4][ref[5].astype(bool)])) > 3  # the masked counts differ between valid nodes
    _check(got, *ref, "oracle")
    per_node = [t.cpu().numpy() for t in K.precompute(d(coords), half, d(f), d(gx), d(gy), d(gz), md, 0.5, 1e12)]
    _check(got, *per_node, "per-node kernel")
    # nodes whose subset leaves the volume: the per-node kernel's outputs exactly
    out = np.zeros(len(coords), dtype=bool)
    out[(coords[:, 0] - 8 < 0) | (coords[:, 0] + 8 >= 64)] = True
    for g_, p_ in zip(got, per_node):
        np.testing.assert_array_equal(g_.cpu().numpy()[out], p_[out])
