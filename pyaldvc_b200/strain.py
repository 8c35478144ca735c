"""Strain after the path, on the device, with the call signatures of pyALDVC's ``al_dvc.strain``.

  gradient_plane_fit, gradient_fd   strain/gradient_methods.py:151-283 (no cut mesh: ``edge_ok`` must be None)
  smooth_grid_field                 utils/grid_interp.py:54-79
  strain_tensor, principal_strains, von_mises_strain, max_shear_strain, volumetric_strain,
  det_deformation_gradient, polar_rotation_deg, scale_to_physical      strain/strain_types.py:19-129
  compute_strain, strain_result_from_gradient                          strain/compute_strain.py:27-145

Functions take host NumPy arrays and return NumPy arrays (the reference's contract); ``compute_strain_device``
is the CUDA-tensor form the pass uses.  Every gradient and strain measure is computed by the library's FP64
kernels (``aldvc_gradient_plane_fit``, ``aldvc_gradient_fd``, ``aldvc_grid_smooth``, ``aldvc_strain_measures``).
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np
import torch

from . import kernels as K


@dataclass
class StrainResult:
    """Strain of one frame (all arrays ``(N,)`` unless stated), fields as the reference's StrainResult."""

    disp_u: np.ndarray
    disp_v: np.ndarray
    disp_w: np.ndarray
    F: np.ndarray  # (N, 3, 3) displacement gradient (physical units)
    exx: np.ndarray
    eyy: np.ndarray
    ezz: np.ndarray
    exy: np.ndarray
    exz: np.ndarray
    eyz: np.ndarray
    principal: np.ndarray  # (N, 3) descending
    max_shear: np.ndarray
    von_mises: np.ndarray
    volumetric: np.ndarray
    det_F: np.ndarray
    rotation_deg: np.ndarray
    strain_valid: np.ndarray
    strain_type: str
    method: str


def _np(t):
    return t.cpu().numpy() if isinstance(t, torch.Tensor) else t


def _no_cut(edge_ok):
    if edge_ok is not None:
        raise NotImplementedError("cut meshes (edge_ok) are not supported by the device strain")


def _grid_valid(U_grid: np.ndarray, valid):
    grid = U_grid.shape[:3]
    ok = np.all(np.isfinite(U_grid), axis=-1)
    if valid is not None:
        ok &= np.asarray(valid, dtype=bool).reshape(grid)
    return ok


def gradient_plane_fit(U_grid, spacing, halfwidth, valid=None, edge_ok=None):
    """Weighted least-squares plane fit of ``U_grid`` (nz, ny, nx, 3) over a (2r+1)^3 node window: returns
    (F_grid (nz, ny, nx, 3, 3), complete (nz, ny, nx)); fewer than 5 valid window nodes -> NaN."""
    _no_cut(edge_ok)
    U = np.asarray(U_grid, dtype=np.float64)
    grid = U.shape[:3]
    v = _grid_valid(U, valid).reshape(-1)
    F, comp = K.gradient_plane_fit(np.ascontiguousarray(U.reshape(-1, 3)), grid, spacing, halfwidth, torch.from_numpy(v))
    return F.cpu().numpy().reshape(grid + (3, 3)), comp.cpu().numpy().reshape(grid)


def gradient_fd(U_grid, spacing, valid=None, edge_ok=None):
    """Central / one-sided finite differences of ``U_grid`` (nz, ny, nx, 3): (F_grid, complete)."""
    _no_cut(edge_ok)
    U = np.asarray(U_grid, dtype=np.float64)
    grid = U.shape[:3]
    v = _grid_valid(U, valid).reshape(-1)
    F, comp = K.gradient_fd(np.ascontiguousarray(U.reshape(-1, 3)), grid, spacing, torch.from_numpy(v))
    return F.cpu().numpy().reshape(grid + (3, 3)), comp.cpu().numpy().reshape(grid)


def smooth_grid_field(field, sigma, valid=None):
    """NaN/mask-aware Gaussian smoothing of a (nz, ny, nx) grid field (sigma in nodes, one value for every axis)."""
    arr = np.array(field, dtype=np.float64, copy=True)
    if sigma is None or (np.isscalar(sigma) and sigma <= 0):
        return arr
    if not np.isscalar(sigma):
        s = tuple(float(x) for x in sigma)
        if len(set(s)) != 1:
            raise NotImplementedError("smooth_grid_field: one sigma for every axis")
        sigma = s[0]
    w = np.isfinite(arr) if valid is None else np.isfinite(arr) & np.asarray(valid, dtype=bool)
    if not w.any():
        return arr
    out = K.grid_smooth(np.ascontiguousarray(arr.reshape(-1)), arr.shape, float(sigma), torch.from_numpy(w.reshape(-1)))
    return out.cpu().numpy().reshape(arr.shape)


def _measures(H, strain_type="infinitesimal") -> dict:
    return K.strain_measures(np.ascontiguousarray(np.asarray(H, dtype=np.float64).reshape(-1, 3, 3)), strain_type)


def deformation_gradient(F_grad):
    return np.asarray(F_grad, dtype=np.float64) + np.eye(3)


def strain_tensor(F_grad, strain_type: str):
    """(N, 3, 3) strain of type infinitesimal, green_lagrange, euler_almansi or hencky."""
    return _np(_measures(F_grad, strain_type)["E"])


def principal_strains(E):
    """Eigenvalues of the symmetric part of E, descending (N, 3)."""
    return _np(_measures(E)["principal"])


def von_mises_strain(E):
    return _np(_measures(E)["von_mises"])


def max_shear_strain(principal):
    p = np.asarray(principal, dtype=np.float64)
    return 0.5 * (p[:, 0] - p[:, 2])


def volumetric_strain(E):
    return np.trace(np.asarray(E, dtype=np.float64), axis1=1, axis2=2)


def det_deformation_gradient(F_grad):
    return _np(_measures(F_grad)["det_F"])


def polar_rotation_deg(F_grad):
    """Rotation angle (degrees) of R in the polar decomposition I + H = R U."""
    return _np(_measures(F_grad)["rotation_deg"])


def scale_to_physical(U, F_grad, voxel_size):
    """u_i^phys = s_i u_i; F_ij^phys = (s_i / s_j) F_ij."""
    s = np.asarray(voxel_size, dtype=np.float64)
    return np.asarray(U, dtype=np.float64) * s[None, :], np.asarray(F_grad, dtype=np.float64) * (s[:, None] / s[None, :])[None]


def _result(U_phys, F_phys, valid, strain_type, method, m) -> StrainResult:
    E = _np(m["E"])
    strain_valid = np.asarray(valid, dtype=bool) & np.all(np.isfinite(E), axis=(1, 2))
    return StrainResult(disp_u=U_phys[:, 0], disp_v=U_phys[:, 1], disp_w=U_phys[:, 2], F=F_phys, exx=E[:, 0, 0], eyy=E[:, 1, 1],
                        ezz=E[:, 2, 2], exy=E[:, 0, 1], exz=E[:, 0, 2], eyz=E[:, 1, 2], principal=_np(m["principal"]),
                        max_shear=_np(m["max_shear"]), von_mises=_np(m["von_mises"]), volumetric=_np(m["volumetric"]),
                        det_F=_np(m["det_F"]), rotation_deg=_np(m["rotation_deg"]), strain_valid=strain_valid, strain_type=strain_type,
                        method=method)


def strain_result_from_gradient(U_phys, F_phys, valid, strain_type: str, method: str) -> StrainResult:
    """Every strain quantity of a frame from its physical displacement (N, 3) and gradient (N, 3, 3)."""
    U_phys = np.asarray(U_phys, dtype=np.float64)
    F_phys = np.asarray(F_phys, dtype=np.float64)
    return _result(U_phys, F_phys, valid, strain_type, method, _measures(F_phys, strain_type))


def compute_strain_device(U, grid_shape, spacing, method: str = "plane_fit", halfwidth=(1, 1, 1), strain_type: str = "infinitesimal",
                          voxel_size=(1.0, 1.0, 1.0), valid=None, F_direct=None, boundary=None, elem_active=None,
                          disp_smoothing: float = 0.0, strain_smoothing: float = 0.0, edge_trim: bool = True, gauss_order: int = 2) -> dict:
    """``compute_strain`` on CUDA tensors: U (N, 3) FP64 in voxels, ``valid`` (N,) bool, ``F_direct`` (N, 3, 3) for
    method "direct", ``boundary`` (N,) bool (grid-surface nodes) for "fem" / "direct" completeness, ``elem_active``
    (E,) uint8 for "fem".  Returns U_phys, F_phys (physical units), the strain measures and ``keep`` (the nodes the
    strain is trusted on)."""
    U = K.dev(U, torch.float64).reshape(-1, 3)
    N = U.shape[0]
    d = U.device
    v = torch.ones(N, dtype=torch.bool, device=d) if valid is None else K.dev(valid, torch.bool).reshape(N)
    v = v & torch.isfinite(U).all(dim=1)
    Ug = torch.where(v[:, None], U, torch.nan)  # the field the gradients see: invalid nodes NaN
    if disp_smoothing > 0:
        Ug = torch.stack([K.grid_smooth(Ug[:, c].contiguous(), grid_shape, disp_smoothing, v) for c in range(3)], 1)
        U = torch.where(v[:, None], Ug, U)  # the reported displacement keeps the raw values of invalid nodes
    if method == "direct" and F_direct is None:
        method = "plane_fit"  # compute_strain.py:64-66
    bnd = torch.zeros(N, dtype=torch.bool, device=d) if boundary is None else K.dev(boundary, torch.bool).reshape(N)
    if method == "plane_fit":
        F, complete = K.gradient_plane_fit(Ug, grid_shape, spacing, halfwidth, v)
    elif method == "fd":
        F, complete = K.gradient_fd(Ug, grid_shape, spacing, v)
    elif method == "fem":
        F = K.nodal_gradient(grid_shape, spacing, elem_active, torch.where(v[:, None], U, 0.0).contiguous(), gauss_order)
        F[~v] = torch.nan
        complete = v & ~bnd
    elif method == "direct":
        F = K.dev(F_direct, torch.float64).reshape(N, 3, 3).clone()
        F[~v] = torch.nan
        complete = v & ~bnd
    else:
        raise ValueError(f"unknown strain_method {method!r}")
    s = torch.as_tensor(np.asarray(voxel_size, dtype=np.float64), device=d)
    U_phys = U * s[None, :]
    F_phys = F * (s[:, None] / s[None, :])[None]
    if strain_smoothing > 0:
        Fs = F_phys.reshape(N, 9)
        F_phys = torch.stack([K.grid_smooth(Fs[:, k].contiguous(), grid_shape, strain_smoothing, v) for k in range(9)], 1).reshape(N, 3, 3)
    keep = v & complete if edge_trim else v
    out = K.strain_measures(F_phys, strain_type)
    out.update(U_phys=U_phys, F_phys=F_phys, keep=keep, method=method)
    return out


def compute_strain(mesh, para, U, F_direct=None, valid=None, ops=None) -> StrainResult:
    """Strain of one frame from the nodal displacement U (N, 3) in voxels (compute_strain.py:27-111): ``mesh`` a
    pyALDVC DVCMesh (grid_shape, spacing, node_valid, boundary_nodes, elements), ``para`` its DVCPara."""
    N = int(mesh.n_nodes)
    grid = tuple(int(g) for g in mesh.grid_shape)
    if hasattr(mesh, "edges_ok_grid"):
        _no_cut(mesh.edges_ok_grid())
    if valid is None:
        valid = mesh.node_valid if np.asarray(mesh.node_valid).size == N else np.ones(N, dtype=bool)
    boundary = np.zeros(N, dtype=bool)
    boundary[np.asarray(mesh.boundary_nodes, dtype=np.int64)] = True
    elem_active = None
    if para.strain_method == "fem":
        elem_active = torch.from_numpy((np.asarray(mesh.elements) >= 0).all(axis=1).astype(np.uint8)).cuda()
    out = compute_strain_device(np.ascontiguousarray(np.asarray(U, dtype=np.float64).reshape(N, 3)), grid, tuple(mesh.spacing),
                                para.strain_method, tuple(para.strain_plane_fit_halfwidth), para.strain_type, tuple(para.voxel_size),
                                torch.from_numpy(np.asarray(valid, dtype=bool).reshape(N)),
                                None if F_direct is None else np.ascontiguousarray(np.asarray(F_direct, dtype=np.float64)),
                                torch.from_numpy(boundary), elem_active, float(para.disp_smoothing), float(para.strain_smoothing),
                                bool(para.strain_edge_trim), int(getattr(para, "gauss_pt_order", 2)))
    return _result(_np(out["U_phys"]), _np(out["F_phys"]), _np(out["keep"]), para.strain_type, out["method"], out)
