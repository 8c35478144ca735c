"""Differentiable ZNSSD residual of warped subsets (torch.autograd.Function over the B200 kernels).

The cost of subset s is C_s = sum_v r_v^2 with r_v = (f_v - mf) / bf - (g(W(x_v; P_s)) - mg) / bg, the
residual pyALDVC's IC-GN minimises (solver/numba_kernels.py:705-708; valid-set statistics :586-598), for the
(2h+1)^3 voxels around node coords[s] and the 12-parameter affine warp P_s = [F row-major, u, v, w].  Forward
and backward are hand-written kernels (``aldvc_znssd_forward`` / ``aldvc_znssd_backward``); the backward
recomputes the interpolation weights and their derivatives instead of storing them, and returns gradients
with respect to P (N,12) and to the deformed volume's voxels.  f, coords, the half-widths and the mode are
constants.
"""

from __future__ import annotations

import torch

from . import kernels as K

MODES = {"linear": 0, "cubic": 1, "bspline": 2}


class ZnssdFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, P, g, f, coords, half, mode):
        cost, stats = K.znssd_forward(f, g, coords, P.detach(), half, mode)
        ctx.save_for_backward(P.detach(), g.detach(), f, coords, stats)
        ctx.half = tuple(int(h) for h in half)
        ctx.mode = int(mode)
        return cost

    @staticmethod
    def backward(ctx, grad_cost):
        P, g, f, coords, stats = ctx.saved_tensors
        need_P, need_g = ctx.needs_input_grad[0], ctx.needs_input_grad[1]
        gP, gG = K.znssd_backward(f, g, coords, P, ctx.half, ctx.mode, stats, grad_cost.contiguous(), need_P, need_g)
        return gP, gG, None, None, None, None


def znssd(P: torch.Tensor, g: torch.Tensor, f: torch.Tensor, coords: torch.Tensor, half, mode="cubic") -> torch.Tensor:
    """ZNSSD cost (N,) FP64 of every subset; differentiable in ``P`` (N,12) FP64 and ``g`` (nz,ny,nx) FP32.

    ``f``, ``g``: CUDA float32 volumes; ``coords``: (N,3) int64 [x, y, z]; ``half``: (hx, hy, hz);
    ``mode``: "linear", "cubic", "bspline" (g holds B-spline coefficients) or 0/1/2.
    """
    m = MODES[mode] if isinstance(mode, str) else int(mode)
    assert f.is_cuda and g.is_cuda and f.dtype == torch.float32 and g.dtype == torch.float32
    return ZnssdFunction.apply(P, g.contiguous(), f.contiguous(), coords.to(torch.int64).contiguous(), tuple(half), m)
