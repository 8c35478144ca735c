"""GPU: strain on the node grid against the reference's own outputs (tests/golden/golden_strain.npz, made by
tests/golden/make_golden.py from strain/compute_strain.py, gradient_methods.py and strain_types.py).

Parity bar: strains within 1e-5 (the target), here held to 1e-9 absolute: both sides are FP64 (the
reference solves its plane-fit normal equations with LAPACK and its 3 x 3 eigen and singular value problems with
numpy, the device with partial-pivoting elimination and Jacobi sweeps); NaN patterns, ``complete`` and
``strain_valid`` flags identical.
"""

from __future__ import annotations

import os
from types import SimpleNamespace

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
TOL = 1e-9
KEYS = ("disp_u", "disp_v", "disp_w", "F", "exx", "eyy", "ezz", "exy", "exz", "eyz", "principal", "max_shear", "von_mises",
        "volumetric", "det_F", "rotation_deg")
CASES = {
    "inf_pf": dict(strain_type="infinitesimal", strain_method="plane_fit"),
    "gl_fd": dict(strain_type="green_lagrange", strain_method="fd"),
    "ea_pf2": dict(strain_type="euler_almansi", strain_method="plane_fit", strain_plane_fit_halfwidth=(2, 1, 1)),
    "he_direct": dict(strain_type="hencky", strain_method="direct", voxel_size=(0.5, 0.7, 1.3)),
    "inf_smooth": dict(strain_type="infinitesimal", strain_method="plane_fit", disp_smoothing=0.8, strain_smoothing=1.1,
                       strain_edge_trim=False),
}


@pytest.fixture(scope="module")
def sg():
    with np.load(os.path.join(HERE, "golden", "golden_strain.npz")) as z:
        return {k: z[k] for k in z.files}


def _mesh(sg):
    x0, y0, z0 = sg["st_x0"], sg["st_y0"], sg["st_z0"]
    grid = (len(z0), len(y0), len(x0))
    return SimpleNamespace(n_nodes=int(np.prod(grid)), grid_shape=grid, spacing=(x0[1] - x0[0], y0[1] - y0[0], z0[1] - z0[0]),
                           node_valid=sg["st_valid"], boundary_nodes=sg["st_boundary"], edges_ok_grid=lambda: None)


def _close(got, ref, what):
    got, ref = np.asarray(got, dtype=np.float64), np.asarray(ref, dtype=np.float64)
    np.testing.assert_array_equal(np.isnan(got), np.isnan(ref), err_msg=f"{what}: NaN pattern")
    np.testing.assert_allclose(np.nan_to_num(got), np.nan_to_num(ref), rtol=0, atol=TOL, err_msg=what)


def test_gradients_match_reference(sg):
    from pyaldvc_b200 import strain as S

    m = _mesh(sg)
    Ug = sg["st_U"].reshape(m.grid_shape + (3,))
    vg = sg["st_valid"].reshape(m.grid_shape)
    for hw in ((1, 1, 1), (2, 1, 1)):
        F, c = S.gradient_plane_fit(Ug, m.spacing, hw, vg)
        tag = f"pf_{hw[0]}{hw[1]}{hw[2]}"
        _close(F, sg[f"{tag}_F"], tag)
        np.testing.assert_array_equal(c, sg[f"{tag}_complete"])
    F, c = S.gradient_fd(Ug, m.spacing, vg)
    _close(F, sg["fd_F"], "fd")
    np.testing.assert_array_equal(c, sg["fd_complete"])


@pytest.mark.parametrize("name", list(CASES))
def test_compute_strain_matches_reference(sg, name):
    from pyaldvc_b200 import strain as S

    para = SimpleNamespace(strain_method="plane_fit", strain_plane_fit_halfwidth=(1, 1, 1), strain_type="infinitesimal",
                           voxel_size=(1.0, 1.0, 1.0), disp_smoothing=0.0, strain_smoothing=0.0, strain_edge_trim=True,
                           gauss_pt_order=2)
    for k, v in CASES[name].items():
        setattr(para, k, v)
    r = S.compute_strain(_mesh(sg), para, sg["st_U"], F_direct=sg["st_F_direct"])
    for k in KEYS:
        _close(getattr(r, k), sg[f"cs_{name}_{k}"], f"{name}.{k}")
    np.testing.assert_array_equal(r.strain_valid, sg[f"cs_{name}_strain_valid"])
    assert r.strain_type == CASES[name]["strain_type"]


def test_strain_measures_of_known_deformations():
    """Closed forms: a rotation by 30 degrees about z has zero Green-Lagrange strain, det 1 and a 30 degree polar
    angle; a reflected stretch keeps its negative det and the rotation of its polar factor; a uniaxial stretch 1.1 gives
    Hencky log(1.1) and Green-Lagrange (1.21 - 1) / 2."""
    from pyaldvc_b200 import strain as S

    t = np.radians(30.0)
    R = np.array([[np.cos(t), -np.sin(t), 0.0], [np.sin(t), np.cos(t), 0.0], [0.0, 0.0, 1.0]])
    # the reflected case has distinct stretches: with equal ones the rotation part of a reflection is not unique
    Hs = np.stack([R - np.eye(3), np.diag([0.1, 0.0, 0.0]), np.diag([1.0, 1.0, -1.0]) @ R @ np.diag([1.1, 1.0, 0.9]) - np.eye(3)])
    gl = S.strain_tensor(Hs, "green_lagrange")
    np.testing.assert_allclose(gl[0], 0.0, atol=1e-15)
    np.testing.assert_allclose(gl[1], np.diag([0.105, 0.0, 0.0]), atol=1e-15)
    np.testing.assert_allclose(S.strain_tensor(Hs[1:2], "hencky")[0], np.diag([np.log(1.1), 0.0, 0.0]), atol=1e-15)
    np.testing.assert_allclose(S.det_deformation_gradient(Hs), [1.0, 1.1, -0.99], atol=1e-15)
    np.testing.assert_allclose(S.polar_rotation_deg(Hs), [30.0, 0.0, 30.0], atol=1e-12)  # the reference gives 30 too
    np.testing.assert_allclose(S.principal_strains(np.stack([np.diag([0.1, -0.2, 0.3])]))[0], [0.3, 0.1, -0.2], atol=1e-15)
