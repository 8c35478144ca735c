"""Automatic choice of the ADMM penalty beta (pyALDVC solver/beta_tuning.py:31-109), on the device.

For every candidate beta_k = beta_range[k] * mean(winstepsize)^2 * mu the global step is solved with zero duals
(``aldvc_global_rhs`` + ``aldvc_pcg_hex8`` + ``aldvc_nodal_gradient``), and Err1 = |U1 - U_hat|,
Err2 = |F1 - grad U_hat| over the included nodes (active, not excluded) are recorded.  The score is the
reference's: "matlab" Err1 + mean(h)^2 Err2 with a discrete minimum, or "normalized" z-scores with a quadratic
refinement in log10(beta).  The five scalars are scored on the host.
"""

from __future__ import annotations

import math

import numpy as np
import torch

from . import kernels as K

# core/config.py:23-30: sqrt(1e-5), 1e-2, sqrt(1e-3), 1e-1, sqrt(1e-1)
DEFAULT_BETA_RANGE = (math.sqrt(1e-5), 1e-2, math.sqrt(1e-3), 1e-1, math.sqrt(1e-1))


def beta_candidates(winstepsize, mu: float, beta_range=DEFAULT_BETA_RANGE) -> np.ndarray:
    """beta_range * mean(winstepsize)^2 * mu (beta_tuning.py:31-33)."""
    h2 = float(np.mean(winstepsize)) ** 2
    return np.asarray(beta_range, dtype=np.float64) * h2 * float(mu)


def active_nodes(grid_shape, elem_active) -> torch.Tensor:
    """(N,) bool: the nodes of at least one active element (all nodes when ``elem_active`` is None)."""
    nz, ny, nx = (int(s) for s in grid_shape)
    if elem_active is None:
        return torch.ones(nz * ny * nx, dtype=torch.bool, device="cuda")
    e = K.dev(elem_active, torch.uint8).reshape(nz - 1, ny - 1, nx - 1) != 0
    a = torch.zeros((nz, ny, nx), dtype=torch.bool, device=e.device)
    for dz in (0, 1):
        for dy in (0, 1):
            for dx in (0, 1):
                a[dz:dz + nz - 1, dy:dy + ny - 1, dx:dx + nx - 1] |= e
    return a.reshape(-1)


def score_sweep(betas, err1, err2, winstepsize, criterion: str = "matlab"):
    """(beta, score, k_best) from the sweep (beta_tuning.py:80-99)."""
    betas, err1, err2 = (np.asarray(a, dtype=np.float64) for a in (betas, err1, err2))
    h2 = float(np.mean(winstepsize)) ** 2
    s1, s2 = np.std(err1), np.std(err2)
    if criterion == "normalized" and s1 > 1e-15 and s2 > 1e-15:
        score = (err1 - err1.mean()) / s1 + (err2 - err2.mean()) / s2
    else:
        score = err1 + err2 * h2
    k_best = int(np.argmin(score))
    beta = float(betas[k_best])
    if criterion == "normalized" and 0 < k_best < len(betas) - 1:
        x = np.log10(betas[k_best - 1:k_best + 2])
        y = score[k_best - 1:k_best + 2]
        p = np.polyfit(x, y, 2)
        if p[0] > 1e-15:
            cand = 10.0 ** (-p[1] / (2.0 * p[0]))
            if betas[k_best - 1] <= cand <= betas[k_best + 1]:
                beta = float(cand)
    return beta, score, k_best


def auto_tune_beta_device(grid_shape, spacing, elem_active, mu: float, alpha: float, U1, F1, exclude=None, winstepsize=(16, 16, 16),
                          beta_range=DEFAULT_BETA_RANGE, criterion: str = "matlab", pcg_tol: float = 1e-8, pcg_max_iter: int = 500,
                          gauss_order: int = 2):
    """Tuned beta and the sweep record; U1 (N, 3), F1 (N, 3, 3) or (N, 9) FP64 CUDA tensors, ``exclude`` (N,) bool."""
    U1 = K.dev(U1, torch.float64).reshape(-1, 3)
    N = U1.shape[0]
    F1 = K.dev(F1, torch.float64).reshape(N, 9)
    betas = beta_candidates(winstepsize, mu, beta_range)
    active = active_nodes(grid_shape, elem_active)
    include = active.clone()
    if exclude is not None:
        ex = K.dev(exclude, torch.bool).reshape(-1)
        if ex.numel() == N:
            include &= ~ex
    if int(include.sum().item()) < 8:
        include = active.clone()
    e = None if elem_active is None else K.dev(elem_active, torch.uint8)
    W0 = torch.zeros((N, 9), dtype=torch.float64, device=U1.device)
    v0 = torch.zeros((N, 3), dtype=torch.float64, device=U1.device)
    err1 = torch.empty(len(betas), dtype=torch.float64, device=U1.device)
    err2 = torch.empty_like(err1)
    words = K.ErrorWords()
    for k, bk in enumerate(betas):
        b = K.global_rhs(grid_shape, spacing, e, float(bk), mu, alpha, U1, F1, W0, v0, gauss_order)
        U2, _, pe = K.pcg_hex8(grid_shape, spacing, e, float(bk), mu, alpha, b, U1, pcg_tol, pcg_max_iter, gauss_order)
        words.add(pe, "pcg_hex8 (beta sweep)")
        F2 = K.nodal_gradient(grid_shape, spacing, e, U2, gauss_order).reshape(N, 9)
        F2 = torch.where(torch.isfinite(F2), F2, F1)
        err1[k] = torch.linalg.vector_norm((U1 - U2)[include])
        err2[k] = torch.linalg.vector_norm((F1 - F2)[include])
    words.check()
    e1, e2 = err1.cpu().numpy(), err2.cpu().numpy()
    beta, score, k_best = score_sweep(betas, e1, e2, winstepsize, criterion)
    return beta, {"betas": betas, "err1": e1, "err2": e2, "score": score, "k_best": k_best, "beta": beta, "criterion": criterion}


def auto_tune_beta(ops, para, mu: float, U1, F1, exclude=None):
    """Host contract of beta_tuning.auto_tune_beta :36-109: ``ops`` a ``subpb2_solver.HexGrid`` (the grid and its
    active elements), ``para`` with winstepsize, beta_range, beta_criterion, alpha, pcg_tol, pcg_max_iter."""
    N = ops.n_nodes
    e = None if ops.elem_active is None else np.ascontiguousarray(ops.elem_active, dtype=np.uint8)
    ex = None if exclude is None else torch.from_numpy(np.asarray(exclude, dtype=bool).reshape(-1))
    return auto_tune_beta_device(ops.grid_shape, ops.spacing, e, float(mu), float(getattr(para, "alpha", 0.0)),
                                 np.ascontiguousarray(np.asarray(U1, dtype=np.float64).reshape(N, 3)),
                                 np.ascontiguousarray(np.asarray(F1, dtype=np.float64).reshape(N, 9)), ex, tuple(para.winstepsize),
                                 tuple(getattr(para, "beta_range", DEFAULT_BETA_RANGE)), getattr(para, "beta_criterion", "matlab"),
                                 float(getattr(para, "pcg_tol", 1e-8)), int(getattr(para, "pcg_max_iter", 500)),
                                 int(getattr(para, "gauss_pt_order", 2)))
