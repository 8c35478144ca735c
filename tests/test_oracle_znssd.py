"""The FP64 ZNSSD cost of the oracle (the checker of the differentiable ZNSSD kernels) against a NumPy
restatement of the reference residual (numba_kernels.py:705-708) built on the oracle's pinned sampler."""

from __future__ import annotations

import numpy as np


def test_oracle_znssd_matches_numpy_residual(oracle_mod):
    from pyaldvc_b200 import synthetic as S

    shape = (40, 40, 40)
    c, pk = S.draw_beads(shape, 0.03, 5)
    f = S.normalize_volume(S.render_beads(shape, c, pk, 1.5))
    g = S.normalize_volume(S.render_beads(shape, S.displace_beads(c, S.translation((0.4, 0.9, -0.6))), pk, 1.5))
    rng = np.random.default_rng(1)
    coords = rng.integers(14, 26, size=(6, 3)).astype(np.int64)
    P = np.zeros((6, 12))
    P[:, :9] = rng.uniform(-0.03, 0.03, size=(6, 9))
    P[:, 9:] = rng.uniform(-1.0, 1.0, size=(6, 3))
    h = 6
    got = oracle_mod.znssd(f, g, coords, P, (h, h, h), 1)
    r = np.arange(-h, h + 1, dtype=np.float64)
    Z, Y, X = (a.ravel() for a in np.meshgrid(r, r, r, indexing="ij"))
    for s in range(len(coords)):
        x0, y0, z0 = coords[s]
        p = P[s]
        xw = (1 + p[0]) * X + p[1] * Y + p[2] * Z + x0 + p[9]
        yw = p[3] * X + (1 + p[4]) * Y + p[5] * Z + y0 + p[10]
        zw = p[6] * X + p[7] * Y + (1 + p[8]) * Z + z0 + p[11]
        gv = oracle_mod.sample_points(g, zw, yw, xw, 1)
        fv = f[(z0 + Z).astype(int), (y0 + Y).astype(int), (x0 + X).astype(int)]
        n = gv.size
        mf = np.sum(fv.astype(np.float64)) / n
        bf = np.sqrt(np.sum((fv * fv).astype(np.float64)) - n * mf * mf)  # float32 squares, as the reference
        mg = gv.mean()
        bg = np.sqrt(np.sum(gv * gv) - n * mg * mg)
        res = (fv.astype(np.float64) - mf) / bf - (gv - mg) / bg
        assert abs(got[s] - np.sum(res * res)) <= 1e-12 * max(1.0, np.sum(res * res))
    # a subset pushed out of the sampler's domain has no cost
    P[0, 9] = 30.0
    assert np.isnan(oracle_mod.znssd(f, g, coords[:1], P[:1], (h, h, h), 1)[0])
