"""CPU: the frame schedule of a series (pyaldvc_b200.frames.FrameSchedule, core/data_structures.py:172-215) and the
node-grid interpolation operators of its cumulative displacements against the reference's interp_grid_field
(tests/golden/golden_series.npz, made by tests/golden/make_golden.py series)."""

from __future__ import annotations

import os
import sys

import numpy as np
import pytest

from pyaldvc_b200.frames import FrameSchedule
from pyaldvc_b200.kernels import spline_axis_operator

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))

import pass_inputs as PI  # noqa: E402


@pytest.fixture(scope="module")
def gs():
    with np.load(os.path.join(HERE, "golden", "golden_series.npz")) as z:
        return {k: z[k] for k in z.files}


def test_schedules():
    assert FrameSchedule.from_mode("accumulative", 4).ref_indices == (0, 0, 0)
    assert FrameSchedule.from_mode("incremental", 4).ref_indices == (0, 1, 2)
    s = FrameSchedule.from_every_n(2, 6)
    assert s.ref_indices == (0, 0, 2, 2, 4) and s.parent(5) == 4
    with pytest.raises(ValueError):
        FrameSchedule((0, 2))  # frame 2 cannot reference frame 2
    with pytest.raises(ValueError):
        FrameSchedule((-1,))
    with pytest.raises(TypeError):
        FrameSchedule((0.0,))
    with pytest.raises(ValueError):
        FrameSchedule.from_mode("sideways", 3)
    with pytest.raises(IndexError):
        FrameSchedule((0, 0)).parent(3)


def test_series_frames_are_the_fixture_frames(gs):
    vols = PI.series_frames()
    assert [PI.sha(v) for v in vols] == [str(s) for s in gs["sha"]]


def _eval(coef, shift, axes, q, order):
    """The device kernel's evaluation (aldvc_grid_interp) restated: weights and taps clamped to the grid."""
    x0, y0, z0 = axes
    h = [a[1] - a[0] if len(a) > 1 else 1.0 for a in (x0, y0, z0)]
    Nz, Ny, Nx = coef.shape
    out = np.empty(len(q))
    for m, p in enumerate(q):
        f = [(p[0] - x0[0]) / h[0] + shift[0], (p[1] - y0[0]) / h[1] + shift[1], (p[2] - z0[0]) / h[2] + shift[2]]
        i0 = [int(np.floor(v)) for v in f]
        t = [v - np.floor(v) for v in f]
        if order == 3:
            w = [np.array([(1 - tt) ** 3, 3 * tt**3 - 6 * tt**2 + 4, -3 * tt**3 + 3 * tt**2 + 3 * tt + 1, tt**3]) / 6 for tt in t]
            taps = [np.clip(np.arange(i - 1, i + 3), 0, n - 1) for i, n in zip(i0, (Nx, Ny, Nz))]
        else:
            w = [np.array([1 - tt, tt]) for tt in t]
            taps = [np.clip(np.arange(i, i + 2), 0, n - 1) for i, n in zip(i0, (Nx, Ny, Nz))]
        sub = coef[np.ix_(taps[2], taps[1], taps[0])]
        out[m] = np.einsum("k,j,i,kji->", w[2], w[1], w[0], sub)
    return out


@pytest.mark.parametrize("gi", range(4))
def test_axis_operators_reproduce_interp_grid_field(gs, gi):
    field, q = gs[f"gi{gi}_field"], gs[f"gi{gi}_q"]
    axes = (gs[f"gi{gi}_x0"], gs[f"gi{gi}_y0"], gs[f"gi{gi}_z0"])
    nz, ny, nx = field.shape
    ox, oy, oz = (spline_axis_operator(n) for n in (nx, ny, nz))
    coef = np.einsum("Xk,zyk->zyX", ox, field)
    coef = np.einsum("Yj,zjX->zYX", oy, coef)
    coef = np.einsum("Zi,iYX->ZYX", oz, coef)
    shift = [(o.shape[0] - n) // 2 for o, n in ((ox, nx), (oy, ny), (oz, nz))]
    np.testing.assert_allclose(_eval(coef, shift, axes, q, 3), gs[f"gi{gi}_o3"], rtol=0, atol=1e-11)
    np.testing.assert_allclose(_eval(field, (0, 0, 0), axes, q, 1), gs[f"gi{gi}_o1"], rtol=0, atol=1e-12)
