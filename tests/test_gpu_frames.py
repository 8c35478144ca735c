"""GPU: frame series (pyaldvc_b200.frames.run_series) against the reference's own run_aldvc over three frames, and
the node-grid interpolation of the cumulative displacements (aldvc_grid_interp) against its interp_grid_field
(tests/golden/golden_series.npz).

Parity bar of the pass (tests/test_gpu_pass.py): displacements within 1e-3 voxel, gradients within 1e-5, identical
statuses, outlier flags and ADMM step counts; the same for the cumulative displacements.  The series driver's own
plumbing (reference cache, previous-frame guess, staged uploads) must not change a pass: every frame equals the
single pass it stands for, bit for bit.
"""

from __future__ import annotations

import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))

import pass_inputs as PI  # noqa: E402

pytestmark = pytest.mark.gpu

U_TOL = 1e-3
F_TOL = 1e-5


@pytest.fixture(scope="module")
def gs():
    with np.load(os.path.join(HERE, "golden", "golden_series.npz")) as z:
        return {k: z[k] for k in z.files}


@pytest.fixture(scope="module")
def vols():
    return PI.series_frames()


def _params(case):
    from pyaldvc_b200.pipeline import PassParams

    c = PI.SERIES_CASES[case]
    return PassParams(**PI.SERIES_PARA, init_guess_method=c["init_guess_method"], global_shift=False, beta=PI.PASS_COMMON["beta"],
                      mu=PI.PASS_COMMON["mu"], autotune=False, threads=128)


@pytest.mark.parametrize("gi", range(4))
def test_grid_interp_matches_interp_grid_field(gs, gi):
    from pyaldvc_b200 import kernels as K

    field, q = gs[f"gi{gi}_field"], gs[f"gi{gi}_q"]
    axes = (gs[f"gi{gi}_x0"], gs[f"gi{gi}_y0"], gs[f"gi{gi}_z0"])
    origin = tuple(float(a[0]) for a in axes)
    h = tuple(float(a[1] - a[0]) if len(a) > 1 else 1.0 for a in axes)
    for order, tol in ((1, 1e-12), (3, 1e-11)):
        got = K.grid_interp(field.reshape(-1), field.shape, origin, h, q, order).cpu().numpy()
        np.testing.assert_allclose(got, gs[f"gi{gi}_o{order}"], rtol=0, atol=tol, err_msg=f"grid {gi} order {order}")


@pytest.mark.parametrize("case", list(PI.SERIES_CASES))
def test_series_matches_reference_run_aldvc(gs, vols, case):
    from pyaldvc_b200.frames import run_series

    c = PI.SERIES_CASES[case]
    res = run_series(vols, _params(case), reference_mode=c["reference_mode"], cumulative_interp=c["cumulative_interp"])
    np.testing.assert_allclose(res.coords, gs[f"{case}_coords"], rtol=0, atol=1e-12)
    assert len(res.frames) == 2
    for k, fr in enumerate(res.frames):
        key = f"{case}_f{k + 1}"
        assert fr.ref_frame == int(gs[f"{key}_ref"]), key
        assert fr.admm_steps == int(gs[f"{key}_steps"]), key
        np.testing.assert_array_equal(fr.status.astype(np.int64), gs[f"{key}_status"].astype(np.int64), err_msg=f"{key} status")
        np.testing.assert_array_equal(fr.outlier, gs[f"{key}_outlier"], err_msg=f"{key} outlier")
        # U_std: the noise model on the final ZNCC and the stored Hessians, about 1e-3 voxel here: 1e-5 is 1 % of it
        for name, tol in (("U0", U_TOL), ("U_local", U_TOL), ("U", U_TOL), ("U_accum", U_TOL), ("F", F_TOL), ("U_std", 1e-5)):
            got = getattr(fr, name).reshape(gs[f"{key}_{name}"].shape)
            np.testing.assert_allclose(got, gs[f"{key}_{name}"], rtol=0, atol=tol, equal_nan=True, err_msg=f"{key} {name}")
    if c["init_guess_method"] == "previous":
        assert res.frames[1].init_method == "previous"
        np.testing.assert_array_equal(res.frames[1].U0, res.frames[0].U)
    if c["reference_mode"] == "incremental":
        assert res.frames[1].ref_frame == 1


def test_series_frames_equal_their_single_passes(vols):
    """Host frames through the staged uploads, the cached reference and the previous-frame guess: every frame is the
    single pass it stands for, bit for bit; the same series from CUDA tensors gives the same frames."""
    import torch

    from pyaldvc_b200.frames import run_series
    from pyaldvc_b200.pipeline import run_pass

    p = _params("accum_prev")
    res = run_series(vols, p)
    cu = [torch.from_numpy(v).cuda() for v in vols]
    one = run_pass(cu[0], cu[1], p)
    two = run_pass(cu[0], cu[2], p, previous=one.U)
    for fr, r in zip(res.frames, (one, two)):
        for k in ("U", "U0", "U_local", "zncc", "status"):
            a, b = getattr(fr, k), getattr(r, k).cpu().numpy()
            assert np.array_equal(a, b, equal_nan=a.dtype.kind == "f"), k
    dev = run_series(cu, p)
    for a, b in zip(res.frames, dev.frames):
        assert np.array_equal(a.U, b.U) and np.array_equal(a.U_accum, b.U_accum)
    assert res.timings["h2d_bytes"] == sum(v.nbytes for v in vols) and dev.timings["h2d_bytes"] == 0


def test_series_strain_is_the_strain_of_the_accumulated_field(vols):
    """Strain per frame (core/pipeline.py:421-433): the device strain of each frame's U_accum on frame 0's node
    grid, the frame's own F for the "direct" method when its reference is frame 0 (the strain module itself is
    pinned to the reference's compute_strain by tests/test_gpu_strain.py)."""
    import torch

    from pyaldvc_b200 import strain as ST
    from pyaldvc_b200.frames import StrainParams, run_series
    from pyaldvc_b200.mesh import surface_nodes

    p = _params("incr_cubic")
    for sp in (StrainParams(), StrainParams(method="direct", strain_type="green_lagrange", voxel_size=(1.0, 1.0, 2.0))):
        res = run_series(vols, p, reference_mode="incremental", strain=sp)
        valid0 = res.frames[0].valid
        bnd = np.zeros(len(valid0), dtype=bool)
        bnd[surface_nodes(res.grid_shape)] = True
        spacing = tuple(float(a[1] - a[0]) for a in res.axes)
        for fr in res.frames:
            out = ST.compute_strain_device(fr.U_accum, res.grid_shape, spacing, sp.method, sp.halfwidth, sp.strain_type, sp.voxel_size,
                                           torch.from_numpy(valid0), fr.F if fr.ref_frame == 0 else None, torch.from_numpy(bnd))
            E = out["E"].cpu().numpy()
            np.testing.assert_array_equal(fr.strain.exx, E[:, 0, 0])
            np.testing.assert_array_equal(fr.strain.eyz, E[:, 1, 2])
            assert fr.strain.method == ("direct" if sp.method == "direct" and fr.ref_frame == 0 else "plane_fit")


def test_tiled_series_equals_resident_series(vols):
    """tile_local > 0: every frame runs the tiled pass from host memory (the reference's tile_local inside run_aldvc);
    the frames equal the resident series' within the tiled pass's own bar (1e-9 voxel), statuses identical."""
    from pyaldvc_b200.frames import run_series

    p = _params("accum_prev")
    p.tile_disp_margin = 2
    whole = run_series(vols, p)
    p.tile_local = 64
    tiled = run_series(vols, p)
    for a, b in zip(whole.frames, tiled.frames):
        np.testing.assert_array_equal(a.status, b.status)
        np.testing.assert_array_equal(a.outlier, b.outlier)
        assert a.init_method == b.init_method and a.admm_steps == b.admm_steps
        for k in ("U0", "U", "U_accum", "U_std"):
            np.testing.assert_allclose(getattr(b, k), getattr(a, k), rtol=0, atol=1e-9, equal_nan=True, err_msg=k)
