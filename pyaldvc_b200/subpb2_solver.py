"""ADMM subproblem 2 on the B200 (pyALDVC solver/subpb2_solver.py:45-155, global_operators.py:58-170).

The reference assembles scipy CSR operators over the active hex8 elements and runs a NumPy PCG.  Here
the operators are never assembled: the mesh is a uniform node grid with a per-element keep flag, and
``aldvc_pcg_hex8`` / ``aldvc_global_rhs`` / ``aldvc_nodal_gradient`` apply the element matrices
matrix-free.  ``GlobalSystem`` / ``build_global_system`` / ``solve_subpb2`` / ``nodal_gradient`` keep
the reference's call shapes for the FEM method with the PCG solver.
"""

from __future__ import annotations

import time
from dataclasses import dataclass

import numpy as np


@dataclass
class HexGrid:
    """Node grid of the global step: ``grid_shape`` (nz, ny, nx), ``spacing`` (x, y, z),
    ``elem_active`` ((nz-1)*(ny-1)*(nx-1),) bool or None for all elements."""

    grid_shape: tuple
    spacing: tuple
    elem_active: np.ndarray | None = None
    gauss_order: int = 2

    @property
    def n_nodes(self) -> int:
        return int(np.prod(self.grid_shape))


@dataclass
class GlobalSystem:
    grid: HexGrid
    beta: float
    mu: float
    alpha: float
    pcg_tol: float = 1e-8
    pcg_max_iter: int = 500
    solver: str = "pcg"
    _elem_d: object = None

    def elem_device(self):
        import torch

        if self.grid.elem_active is None:
            return None
        if self._elem_d is None:
            self._elem_d = torch.from_numpy(np.ascontiguousarray(self.grid.elem_active, dtype=np.uint8)).cuda()
        return self._elem_d


def build_global_system(grid: HexGrid, beta: float, mu: float, alpha: float = 0.0, pcg_tol: float = 1e-8,
                        pcg_max_iter: int = 500) -> GlobalSystem:
    """``A = (beta + alpha) Kg + mu M`` on the active nodes (subpb2_solver.build_global_system :45-74, PCG)."""
    return GlobalSystem(grid, float(beta), float(mu), float(alpha), float(pcg_tol), int(pcg_max_iter))


def _kernels():
    from .cuda_kernels import _require

    return _require()


def solve_subpb2_device(system: GlobalSystem, U1, F1, W, v):
    """Device tensors in and out: returns (U2 (N,3), iters (device int32), err (device int32))."""
    K = _kernels()
    g = system.grid
    e = system.elem_device()
    b = K.global_rhs(g.grid_shape, g.spacing, e, system.beta, system.mu, system.alpha, U1, F1, W, v, g.gauss_order)
    return K.pcg_hex8(g.grid_shape, g.spacing, e, system.beta, system.mu, system.alpha, b, U1, system.pcg_tol,
                      system.pcg_max_iter, g.gauss_order)


def solve_subpb2(system: GlobalSystem, U1, F1, W, v):
    """``u_hat`` (N, 3); inactive nodes keep ``U1`` (subpb2_solver.solve_subpb2 :133-155)."""
    t0 = time.perf_counter()
    U2, iters, err = solve_subpb2_device(system, U1, F1, W, v)
    words = _kernels().ErrorWords()
    words.add(err, "pcg_hex8")
    words.check()
    info = {"solver": "pcg", "iterations": int(iters.item()), "time": time.perf_counter() - t0}
    return U2.cpu().numpy(), info


def global_rhs(system: GlobalSystem, U1, F1, W, v) -> np.ndarray:
    K = _kernels()
    g = system.grid
    return K.global_rhs(g.grid_shape, g.spacing, system.elem_device(), system.beta, system.mu, system.alpha, U1, F1, W, v,
                        g.gauss_order).cpu().numpy()


def nodal_gradient(system_or_grid, U) -> np.ndarray:
    """``(N, 3, 3)`` F_ij = (G_j^T u_i) / m_L, NaN off the active set (global_operators.nodal_gradient :151-170)."""
    K = _kernels()
    if isinstance(system_or_grid, GlobalSystem):
        g, e = system_or_grid.grid, system_or_grid.elem_device()
    else:
        import torch

        g = system_or_grid
        e = None if g.elem_active is None else torch.from_numpy(np.ascontiguousarray(g.elem_active, np.uint8)).cuda()
    return K.nodal_gradient(g.grid_shape, g.spacing, e, U, g.gauss_order).cpu().numpy()
