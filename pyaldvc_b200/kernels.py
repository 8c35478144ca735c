"""Device-level API: torch CUDA tensors in, torch CUDA tensors out, every call through the C ABI.

PyTorch provides device memory, the current stream and the caching allocator for workspaces;
the arithmetic is the library's.  All calls are stream-ordered on ``torch.cuda.current_stream()``
and return without synchronising, so they can be chained (and captured in a CUDA graph).
"""

from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib

BATCHED = _lib.BATCHED
PLAIN = _lib.PLAIN
NCC_TILED = _lib.NCC_TILED
NCC_PLAIN = _lib.NCC_PLAIN
NCC_FFT = _lib.NCC_FFT
NCC_FFT_STOCKHAM = _lib.NCC_FFT_STOCKHAM
NCC_FFT_CLUSTER = _lib.NCC_FFT_CLUSTER
INTERP_MODE_BY_NAME = {"linear": 0, "cubic": 1, "bspline": 2}


def lib():
    return _lib.load()


def stream_handle() -> int:
    return torch.cuda.current_stream().cuda_stream


def dev(a, dtype: torch.dtype) -> torch.Tensor:
    """A contiguous CUDA tensor of ``dtype`` (host arrays are copied)."""
    if isinstance(a, torch.Tensor):
        t = a if a.is_cuda else a.to("cuda", non_blocking=False)
        t = t.to(dtype) if t.dtype != dtype else t
        return t.contiguous()
    return torch.from_numpy(np.ascontiguousarray(a)).to(device="cuda", dtype=dtype)


def _p(t: torch.Tensor | None):
    return None if t is None else ctypes.c_void_p(t.data_ptr())


def _workspace(nbytes: int) -> torch.Tensor:
    return torch.empty(max(int(nbytes), 256), dtype=torch.uint8, device="cuda")


def volumes_struct(f, gx, gy, gz, mask, g, g4=None) -> _lib.Volumes:
    nz, ny, nx = f.shape
    return _lib.Volumes(f.data_ptr(), None if gx is None else gx.data_ptr(), None if gy is None else gy.data_ptr(),
                        None if gz is None else gz.data_ptr(), None if mask is None else mask.data_ptr(),
                        None if g is None else g.data_ptr(), nz, ny, nx, None if g4 is None else g4.data_ptr())


def make_quads(vol: torch.Tensor) -> torch.Tensor:
    """(n, 4) float32 overlapping quads of a float32 CUDA volume: row i holds vol[i], vol[i+1], vol[i+2], vol[i+3]
    (clamped at the end): the IC-GN kernels read a cubic tap row with one 16-byte load from it."""
    vol = dev(vol, torch.float32)
    q = torch.empty((vol.numel(), 4), dtype=torch.float32, device=vol.device)
    _lib.check(lib().aldvc_make_quads(_p(vol), vol.numel(), _p(q), stream_handle()), "aldvc_make_quads")
    return q


def subset_struct(half, stride, mode, split_index=None, split_keep=None, node_half=None) -> _lib.Subset:
    """``half`` (hx, hy, hz); with ``node_half`` ((N,3) int32 CUDA tensor of per-node half-widths) ``half`` must be
    their maximum."""
    hx, hy, hz = (int(h) for h in half)
    nh = None if node_half is None else node_half.data_ptr()
    if split_index is not None and split_keep is not None:
        return _lib.Subset(hx, hy, hz, int(stride), int(mode), 0, split_index.data_ptr(), split_keep.data_ptr(),
                           int(split_keep.shape[1]), nh)
    return _lib.Subset(hx, hy, hz, int(stride), int(mode), 0, None, None, 0, nh)


# --------------------------------------------------------------------------- preprocessing
def gradients(f: torch.Tensor, border: int = 3):
    """Stencil-7 gradients of a (nz, ny, nx) float32 CUDA volume."""
    f = dev(f, torch.float32)
    gx, gy, gz = (torch.empty_like(f) for _ in range(3))
    nz, ny, nx = f.shape
    _lib.check(lib().aldvc_gradients(_p(f), nz, ny, nx, int(border), _p(gx), _p(gy), _p(gz), stream_handle()),
               "aldvc_gradients")
    return gx, gy, gz


# --------------------------------------------------------------------------- local solver
def precompute(coords, half, f, gx, gy, gz, mask, min_valid_ratio, cond_max, stride=1, split_index=None, split_keep=None,
               node_half=None):
    """Device ``precompute_nodes``: returns (H (N,12,12), L (N,12,12), meanf, bottomf, n_valid, valid) tensors.
    ``node_half``: optional (N,3) per-node half-widths (uneven subsets; ``half`` is then their maximum)."""
    coords = dev(coords, torch.int64)
    N = coords.shape[0]
    d = coords.device
    H = torch.empty((N, 12, 12), dtype=torch.float64, device=d)
    L = torch.empty((N, 12, 12), dtype=torch.float64, device=d)
    mf = torch.empty(N, dtype=torch.float64, device=d)
    bf = torch.empty(N, dtype=torch.float64, device=d)
    nv = torch.empty(N, dtype=torch.int64, device=d)
    valid = torch.empty(N, dtype=torch.uint8, device=d)
    vol = volumes_struct(f, gx, gy, gz, mask, None)
    nh = None if node_half is None else dev(node_half, torch.int32)
    sub = subset_struct(half, stride, 0, split_index, split_keep, nh)
    _lib.check(lib().aldvc_precompute(ctypes.byref(vol), ctypes.byref(sub), _p(coords), N, float(min_valid_ratio),
                                      float(cond_max), _p(H), _p(L), _p(mf), _p(bf), _p(nv), _p(valid), stream_handle()),
               "aldvc_precompute")
    return H, L, mf, bf, nv, valid


def precompute_grid(xs, ys, zs, half, f, gx, gy, gz, min_valid_ratio, cond_max, mask=None):
    """``precompute`` for the nodes of the tensor grid xs x ys x zs (node (iz * ny + iy) * nx + ix), separable sums;
    stored gradients, optional uint8 mask, stride 1.  Same outputs as ``precompute``."""
    xs, ys, zs = (dev(np.asarray(a, dtype=np.int64) if not isinstance(a, torch.Tensor) else a, torch.int64).reshape(-1)
                  for a in (xs, ys, zs))
    N = xs.numel() * ys.numel() * zs.numel()
    d = f.device
    H = torch.empty((N, 12, 12), dtype=torch.float64, device=d)
    L = torch.empty((N, 12, 12), dtype=torch.float64, device=d)
    mf = torch.empty(N, dtype=torch.float64, device=d)
    bf = torch.empty(N, dtype=torch.float64, device=d)
    nv = torch.empty(N, dtype=torch.int64, device=d)
    valid = torch.empty(N, dtype=torch.uint8, device=d)
    m = None if mask is None else dev(mask, torch.uint8)
    vol = volumes_struct(f, gx, gy, gz, m, None)
    sub = subset_struct(half, 1, 0, None, None, None)
    nz, ny, nx = f.shape
    ws = _workspace(lib().aldvc_precompute_grid_workspace_size(nz, ny, nx, xs.numel(), ys.numel()))
    _lib.check(lib().aldvc_precompute_grid(ctypes.byref(vol), ctypes.byref(sub), _p(xs), xs.numel(), _p(ys), ys.numel(), _p(zs),
                                           zs.numel(), float(min_valid_ratio), float(cond_max), _p(H), _p(L), _p(mf), _p(bf), _p(nv),
                                           _p(valid), _p(ws), ws.numel(), stream_handle()), "aldvc_precompute_grid")
    return H, L, mf, bf, nv, valid


def icgn_params(tol, dp_tol, max_iter, patience, noise_gain=0.0, predictive=True, variant=BATCHED, threads=0, brick_floats=0,
                mu=0.0, n_full=0.0, sweep_rows=0, node_order=None) -> _lib.IcgnParams:
    """``node_order``: optional (N,) int32 CUDA tensor, the permutation the persistent work queue follows."""
    return _lib.IcgnParams(float(tol), float(dp_tol), int(max_iter), int(patience), float(noise_gain), int(bool(predictive)),
                           int(variant), int(threads), int(brick_floats), float(mu), float(n_full), int(sweep_rows), 0,
                           None if node_order is None else node_order.data_ptr())


def icgn12(coords, P0, half, f, gx, gy, gz, mask, g, mode, L, meanf, valid, tol, dp_tol, max_iter, patience, stride=1, H=None,
           pattern=None, noise_gain=0.0, predictive=True, split_index=None, split_keep=None, variant=BATCHED, threads=0,
           brick_floats=0, node_half=None, g4=None, sweep_rows=0, node_order=None, errs=None):
    """Device 12-DOF IC-GN; returns (P (N,12), n_iter, status, zncc) tensors.  ``node_half``: optional (N,3)
    per-node half-widths (``half`` is then their maximum); ``sweep_rows``: rows per sweep tile of the persistent
    form (0 library default, < 0 C order); ``threads`` 128 with ``brick_floats`` -1: the persistent sweep staged
    through TMA copies of g; ``errs`` (an ErrorWords) receives the launch's device error word."""
    coords = dev(coords, torch.int64)
    N = coords.shape[0]
    d = coords.device
    P0 = dev(P0, torch.float64).reshape(N, 12)
    P = torch.empty((N, 12), dtype=torch.float64, device=d)
    n_iter = torch.empty(N, dtype=torch.int32, device=d)
    status = torch.empty(N, dtype=torch.int8, device=d)
    zncc = torch.empty(N, dtype=torch.float64, device=d)
    vol = volumes_struct(f, gx, gy, gz, mask, g, g4)
    nh = None if node_half is None else dev(node_half, torch.int32)
    sub = subset_struct(half, stride, mode, split_index, split_keep, nh)
    order = None if node_order is None else dev(node_order, torch.int32)
    prm = icgn_params(tol, dp_tol, max_iter, patience, noise_gain, predictive, variant, threads, brick_floats, sweep_rows=sweep_rows,
                      node_order=order)
    ws_n = lib().aldvc_icgn_workspace_size(ctypes.byref(sub), N, ctypes.byref(prm))
    ws = _workspace(ws_n)
    use_noise = noise_gain > 0.0 and H is not None and pattern is not None
    Hd = dev(H, torch.float64) if use_noise else None
    pat = dev(pattern, torch.float64) if use_noise else None
    _lib.check(lib().aldvc_icgn12(ctypes.byref(vol), ctypes.byref(sub), _p(coords), N, _p(P0), _p(L), _p(Hd), _p(pat), _p(meanf),
                                  _p(valid), ctypes.byref(prm), _p(ws), ws.numel(), _p(P), _p(n_iter), _p(status), _p(zncc),
                                  stream_handle()), "aldvc_icgn12")
    if errs is not None and variant == BATCHED:
        errs.add(ws[:8].view(torch.int32)[1:2], "icgn12")  # the word after the work counter
    return P, n_iter, status, zncc


def icgn3(coords, U_old, F_fixed, vdual, half, f, gx, gy, gz, mask, g, mode, H, meanf, bottomf, valid, mu, tol, dp_tol, max_iter,
          patience, stride=1, n_full=0.0, noise_gain=0.0, predictive=True, split_index=None, split_keep=None, variant=BATCHED,
          threads=0, brick_floats=0, node_half=None, g4=None, sweep_rows=0, node_order=None, errs=None):
    """Device 3-DOF IC-GN (ADMM subproblem 1); returns (U (N,3), n_iter, status, zncc) tensors (arguments as icgn12)."""
    coords = dev(coords, torch.int64)
    N = coords.shape[0]
    d = coords.device
    U_old = dev(U_old, torch.float64).reshape(N, 3)
    F_fixed = dev(F_fixed, torch.float64).reshape(N, 9)
    vdual = dev(vdual, torch.float64).reshape(N, 3)
    U = torch.empty((N, 3), dtype=torch.float64, device=d)
    n_iter = torch.empty(N, dtype=torch.int32, device=d)
    status = torch.empty(N, dtype=torch.int8, device=d)
    zncc = torch.empty(N, dtype=torch.float64, device=d)
    vol = volumes_struct(f, gx, gy, gz, mask, g, g4)
    nh = None if node_half is None else dev(node_half, torch.int32)
    sub = subset_struct(half, stride, mode, split_index, split_keep, nh)
    order = None if node_order is None else dev(node_order, torch.int32)
    prm = icgn_params(tol, dp_tol, max_iter, patience, noise_gain, predictive, variant, threads, brick_floats, mu, n_full,
                      sweep_rows, order)
    ws = _workspace(lib().aldvc_icgn_workspace_size(ctypes.byref(sub), N, ctypes.byref(prm)))
    _lib.check(lib().aldvc_icgn3(ctypes.byref(vol), ctypes.byref(sub), _p(coords), N, _p(U_old), _p(F_fixed), _p(vdual), _p(H),
                                 _p(meanf), _p(bottomf), _p(valid), ctypes.byref(prm), _p(ws), ws.numel(), _p(U), _p(n_iter),
                                 _p(status), _p(zncc), stream_handle()), "aldvc_icgn3")
    if errs is not None and variant == BATCHED:
        errs.add(ws[:8].view(torch.int32)[1:2], "icgn3")
    return U, n_iter, status, zncc


# --------------------------------------------------------------------------- integer search
def ncc_map(f, g, coords, half, radius, wx0, wy0, wz0, t_ok) -> torch.Tensor:
    """Device ``_zncc_direct``: (N, 2rz+1, 2ry+1, 2rx+1) float32 maps."""
    coords = dev(coords, torch.int64)
    N = coords.shape[0]
    hx, hy, hz = (int(h) for h in half)
    rx, ry, rz = (int(r) for r in radius)
    out = torch.empty((N, 2 * rz + 1, 2 * ry + 1, 2 * rx + 1), dtype=torch.float32, device=coords.device)
    wx0, wy0, wz0 = (dev(a, torch.int64) for a in (wx0, wy0, wz0))
    t_ok = dev(t_ok, torch.uint8)
    nz, ny, nx = f.shape
    _lib.check(lib().aldvc_ncc_map(_p(f), _p(g), nz, ny, nx, _p(coords), N, hx, hy, hz, rx, ry, rz, _p(wx0), _p(wy0), _p(wz0),
                                   _p(t_ok), _p(out), stream_handle()), "aldvc_ncc_map")
    return out


def ncc_search(f, g, coords, half, radius, shift0=None, engine: int = _lib.NCC_TILED) -> dict:
    """Device single-level search; returns dict of tensors disp (N,3), cc, pce, clipped, ok.
    ``engine``: NCC_TILED (default), NCC_PLAIN or NCC_FFT."""
    coords = dev(coords, torch.int64)
    N = coords.shape[0]
    d = coords.device
    hx, hy, hz = (int(h) for h in half)
    rx, ry, rz = (int(r) for r in radius)
    sh = None if shift0 is None else dev(shift0, torch.int64).reshape(N, 3)
    disp = torch.empty((N, 3), dtype=torch.float64, device=d)
    cc = torch.empty(N, dtype=torch.float64, device=d)
    pce = torch.empty(N, dtype=torch.float64, device=d)
    clipped = torch.empty(N, dtype=torch.uint8, device=d)
    ok = torch.empty(N, dtype=torch.uint8, device=d)
    nz, ny, nx = f.shape
    ws = _workspace(lib().aldvc_ncc_search_workspace_size(nz, ny, nx, N, hx, hy, hz, rx, ry, rz, int(engine)))
    _lib.check(lib().aldvc_ncc_search(_p(f), _p(g), nz, ny, nx, _p(coords), N, hx, hy, hz, rx, ry, rz, _p(sh), int(engine),
                                      _p(ws), ws.numel(), _p(disp), _p(cc), _p(pce), _p(clipped), _p(ok), stream_handle()),
               "aldvc_ncc_search")
    return {"disp": disp, "cc": cc, "pce": pce, "clipped": clipped, "ok": ok}


# --------------------------------------------------------------------------- global step
def mesh_struct(grid_shape, spacing, elem_active=None, gauss_order=2) -> _lib.Hex8Mesh:
    nz, ny, nx = (int(s) for s in grid_shape)
    sx, sy, sz = (float(s) for s in spacing)
    return _lib.Hex8Mesh(nx, ny, nz, sx, sy, sz, None if elem_active is None else elem_active.data_ptr(), int(gauss_order), 0)


def global_rhs(grid_shape, spacing, elem_active, beta, mu, alpha, U1, F1, W, v, gauss_order=2) -> torch.Tensor:
    U1 = dev(U1, torch.float64).reshape(-1, 3)
    N = U1.shape[0]
    F1, W = (dev(a, torch.float64).reshape(N, 9) for a in (F1, W))
    v = dev(v, torch.float64).reshape(N, 3)
    b = torch.empty((N, 3), dtype=torch.float64, device=U1.device)
    m = mesh_struct(grid_shape, spacing, elem_active, gauss_order)
    _lib.check(lib().aldvc_global_rhs(ctypes.byref(m), float(beta), float(mu), float(alpha), _p(U1), _p(F1), _p(W), _p(v), _p(b),
                                      stream_handle()), "aldvc_global_rhs")
    return b


def pcg_hex8(grid_shape, spacing, elem_active, beta, mu, alpha, B, X0, tol, max_iter, gauss_order=2):
    """Jacobi-PCG on the hex8 system; returns (X (N,3), iters (device int32), err (device int32))."""
    B = dev(B, torch.float64).reshape(-1, 3)
    X0 = dev(X0, torch.float64).reshape(-1, 3)
    X = torch.empty_like(B)
    iters = torch.zeros(1, dtype=torch.int32, device=B.device)
    err = torch.zeros(1, dtype=torch.int32, device=B.device)
    m = mesh_struct(grid_shape, spacing, elem_active, gauss_order)
    ws = _workspace(lib().aldvc_pcg_workspace_size(ctypes.byref(m)))
    _lib.check(lib().aldvc_pcg_hex8(ctypes.byref(m), float(beta), float(mu), float(alpha), _p(B), _p(X0), float(tol), int(max_iter),
                                    _p(ws), ws.numel(), _p(X), _p(iters), _p(err), stream_handle()), "aldvc_pcg_hex8")
    return X, iters, err


def nodal_gradient(grid_shape, spacing, elem_active, U, gauss_order=2) -> torch.Tensor:
    U = dev(U, torch.float64).reshape(-1, 3)
    F = torch.empty((U.shape[0], 3, 3), dtype=torch.float64, device=U.device)
    m = mesh_struct(grid_shape, spacing, elem_active, gauss_order)
    _lib.check(lib().aldvc_nodal_gradient(ctypes.byref(m), _p(U), _p(F), stream_handle()), "aldvc_nodal_gradient")
    return F


# --------------------------------------------------------------------------- device error words
class DeviceError(RuntimeError):
    """A bounded device-side wait gave up: a grid barrier of a cooperative kernel (PCG, inpainting) whose peer
    blocks did not arrive within the spin limit.  The kernel set its error word and returned; its output is
    not a solution."""


class ErrorWords:
    """The device error words of a sequence of launches, read once at the end: ``add`` keeps the word (no
    synchronisation), ``check`` reduces every word on the device, reads one scalar and raises DeviceError
    naming the launches that gave up."""

    def __init__(self):
        self.words: list = []
        self.names: list = []

    def add(self, err, what: str) -> None:
        self.words.append(err.reshape(-1)[:1])
        self.names.append(what)

    def extend(self, other: "ErrorWords") -> None:
        self.words += other.words
        self.names += other.names

    def check(self) -> None:
        if not self.words:
            return
        flags = torch.cat(self.words)
        if int(flags.max().item()) == 0:
            return
        bad = sorted({n for n, v in zip(self.names, flags.cpu().tolist()) if v != 0})
        raise DeviceError(f"a bounded device wait gave up in {', '.join(bad)} (grid barrier spin limit reached)")


def test_set_barrier(extra_arrivals: int = 0, spin_limit: int = 0) -> None:
    """Test hook of the bounded grid barriers (aldvc_test_set_barrier): the cooperative kernels wait for
    ``extra_arrivals`` more blocks than they launch and give up after ``spin_limit`` polls; (0, 0) restores
    the production barrier."""
    _lib.check(lib().aldvc_test_set_barrier(int(extra_arrivals), int(spin_limit)), "aldvc_test_set_barrier")


# --------------------------------------------------------------------------- kernel timing
def kernel_timing(enable: bool) -> None:
    """Start (clearing earlier records) or stop the library's per-launch CUDA-event timing of its main kernels."""
    _lib.check(lib().aldvc_kernel_timing(1 if enable else 0), "aldvc_kernel_timing")


def kernel_timing_read(max_entries: int = 64) -> dict:
    """{kernel name: (total device ms, launches)} of the launches recorded since timing started."""
    name_len = 48
    names = ctypes.create_string_buffer(max_entries * name_len)
    ms = (ctypes.c_double * max_entries)()
    cnt = (ctypes.c_int64 * max_entries)()
    n = lib().aldvc_kernel_timing_read(max_entries, names, name_len, ms, cnt)
    if n < 0:
        _lib.check(n, "aldvc_kernel_timing_read")
    out = {}
    for i in range(min(n, max_entries)):
        nm = names.raw[i * name_len:(i + 1) * name_len].split(b"\0", 1)[0].decode()
        out[nm] = (float(ms[i]), int(cnt[i]))
    return out


# --------------------------------------------------------------------------- differentiable ZNSSD residual
ZNSSD_STATS = 7


def znssd_forward(f, g, coords, P, half, mode) -> tuple[torch.Tensor, torch.Tensor]:
    """ZNSSD cost (N,) FP64 of every subset under its warp P (N,12) FP64, and the (N,7) statistics the
    backward needs."""
    coords = dev(coords, torch.int64)
    P = dev(P, torch.float64).reshape(-1, 12)
    n = coords.shape[0]
    cost = torch.empty(n, dtype=torch.float64, device=P.device)
    stats = torch.empty((n, ZNSSD_STATS), dtype=torch.float64, device=P.device)
    vol = volumes_struct(f, None, None, None, None, g)
    hx, hy, hz = (int(h) for h in half)
    _lib.check(lib().aldvc_znssd_forward(ctypes.byref(vol), _p(coords), n, hx, hy, hz, int(mode), _p(P), _p(cost), _p(stats),
                                         stream_handle()), "aldvc_znssd_forward")
    return cost, stats


def znssd_backward(f, g, coords, P, half, mode, stats, grad_cost, need_P=True, need_g=True):
    """Gradients of sum_s grad_cost[s] C_s with respect to P (N,12) and to the voxels of g (nz,ny,nx) FP32."""
    coords = dev(coords, torch.int64)
    P = dev(P, torch.float64).reshape(-1, 12)
    grad_cost = dev(grad_cost, torch.float64).reshape(-1).contiguous()
    n = coords.shape[0]
    gP = torch.empty((n, 12), dtype=torch.float64, device=P.device) if need_P else None
    gG = torch.zeros_like(g) if need_g else None
    vol = volumes_struct(f, None, None, None, None, g)
    hx, hy, hz = (int(h) for h in half)
    _lib.check(lib().aldvc_znssd_backward(ctypes.byref(vol), _p(coords), n, hx, hy, hz, int(mode), _p(P), _p(stats), _p(grad_cost),
                                          None if gP is None else _p(gP), None if gG is None else _p(gG), stream_handle()),
               "aldvc_znssd_backward")
    return gP, gG


# --------------------------------------------------------------------------- volumes and node-grid post-processing
def normalize(vol: torch.Tensor, pilot: float | None = None) -> torch.Tensor:
    """``(vol - mean) / std`` of a float32 or uint16 CUDA volume as float32 (FP64 statistics)."""
    assert vol.is_cuda and vol.is_contiguous()
    if vol.dtype == torch.uint16:
        is16 = 1
    elif vol.dtype == torch.float32:
        is16 = 0
    else:
        raise TypeError("normalize: float32 or uint16 volume")
    if pilot is None:  # the reference's pilot: the centre voxel (io/volume_ops.py:94-99)
        nz, ny, nx = vol.shape
        pilot = float(vol[nz // 2, ny // 2, nx // 2].item())
    out = torch.empty(vol.shape, dtype=torch.float32, device=vol.device)
    ws = _workspace(lib().aldvc_normalize_workspace_size())
    _lib.check(lib().aldvc_normalize(_p(vol), is16, vol.numel(), float(pilot), _p(out), None, _p(ws), ws.numel(),
                                     stream_handle()), "aldvc_normalize")
    return out


def _vol_kind(vol: torch.Tensor) -> int:
    if vol.dtype == torch.uint16:
        return 1
    if vol.dtype == torch.float32:
        return 0
    raise TypeError("float32 or uint16 volume expected")


def _box(box):
    if box is None:
        return None
    b = (ctypes.c_int64 * 6)(*(int(v) for v in box))
    return ctypes.cast(b, ctypes.c_void_p), b  # keep the array alive with the pointer


def _box_pilot(vol: torch.Tensor, box) -> float:
    """The reference's pilot value: the centre voxel of the box (io/volume_ops.py:86)."""
    nz, ny, nx = vol.shape
    z0, z1, y0, y1, x0, x1 = box if box is not None else (0, nz, 0, ny, 0, nx)
    return float(vol[(z0 + z1) // 2, (y0 + y1) // 2, (x0 + x1) // 2].item())


def volume_stats(vol: torch.Tensor, box=None, pilot: float | None = None) -> torch.Tensor:
    """(mean, population std) FP64 device tensor of a float32/uint16 CUDA volume over ``box`` =
    (z0, z1, y0, y1, x0, x1) half-open (None: whole volume)."""
    assert vol.is_cuda and vol.is_contiguous()
    kind = _vol_kind(vol)
    if pilot is None:
        pilot = _box_pilot(vol, box)
    stats = torch.empty(2, dtype=torch.float64, device=vol.device)
    ws = _workspace(lib().aldvc_stats_workspace_size())
    bp = _box(box)
    nz, ny, nx = vol.shape
    _lib.check(lib().aldvc_volume_stats(_p(vol), kind, nz, ny, nx, None if bp is None else bp[0], float(pilot), _p(stats), _p(ws),
                                        ws.numel(), stream_handle()), "aldvc_volume_stats")
    return stats


def normalize_voi(vol: torch.Tensor, box, pilot: float | None = None):
    """(v - mean) / std of the whole volume with the statistics of ``box``; returns (float32 volume, stats)."""
    assert vol.is_cuda and vol.is_contiguous()
    kind = _vol_kind(vol)
    if pilot is None:
        pilot = _box_pilot(vol, box)
    out = torch.empty(vol.shape, dtype=torch.float32, device=vol.device)
    stats = torch.empty(2, dtype=torch.float64, device=vol.device)
    ws = _workspace(lib().aldvc_stats_workspace_size())
    bp = _box(box)
    nz, ny, nx = vol.shape
    _lib.check(lib().aldvc_normalize_voi(_p(vol), kind, nz, ny, nx, None if bp is None else bp[0], float(pilot), _p(out), _p(stats),
                                         _p(ws), ws.numel(), stream_handle()), "aldvc_normalize_voi")
    return out, stats


def volume_moments(vol: torch.Tensor, pilot: float, sums: torch.Tensor) -> torch.Tensor:
    """Add the FP64 sums of (v - pilot) and (v - pilot)^2 of a float32 / uint16 CUDA array into ``sums`` (2 doubles,
    device): the moments of a volume streamed through the device slab by slab."""
    assert vol.is_cuda and vol.is_contiguous() and sums.dtype == torch.float64 and sums.numel() == 2
    ws = _workspace(lib().aldvc_normalize_workspace_size())
    _lib.check(lib().aldvc_volume_moments(_p(vol), _vol_kind(vol), vol.numel(), float(pilot), _p(sums), _p(ws), ws.numel(),
                                          stream_handle()), "aldvc_volume_moments")
    return sums


def normalize_sums(vol: torch.Tensor, sums: torch.Tensor, n_total: int, pilot: float) -> torch.Tensor:
    """(v - mean) / std of a float32 / uint16 CUDA array as float32, mean and std from the accumulated ``sums`` of a
    volume of ``n_total`` voxels about ``pilot`` (one box of a streamed volume, the whole volume's statistics)."""
    assert vol.is_cuda and vol.is_contiguous() and sums.dtype == torch.float64 and sums.numel() == 2
    out = torch.empty(vol.shape, dtype=torch.float32, device=vol.device)
    _lib.check(lib().aldvc_normalize_sums(_p(vol), _vol_kind(vol), vol.numel(), _p(sums), int(n_total), float(pilot), _p(out), None,
                                          stream_handle()), "aldvc_normalize_sums")
    return out


def block_downsample(vol: torch.Tensor, factor: int) -> torch.Tensor:
    """Block means of ``factor``^3 voxels (trailing voxels dropped); ``factor <= 1`` returns a float32 copy."""
    vol = dev(vol, torch.float32)
    if factor <= 1:
        return vol.clone()
    nz, ny, nx = vol.shape
    out = torch.empty((nz // factor, ny // factor, nx // factor), dtype=torch.float32, device=vol.device)
    _lib.check(lib().aldvc_block_downsample(_p(vol), nz, ny, nx, int(factor), _p(out), stream_handle()), "aldvc_block_downsample")
    return out


def phase_correlation_peak(fs: torch.Tensor, gs: torch.Tensor) -> tuple:
    """(pz, py, px): the first maximum of the phase-correlation surface of two equal-shape float32 CUDA volumes."""
    fs = dev(fs, torch.float32)
    gs = dev(gs, torch.float32)
    if fs.shape != gs.shape:
        raise ValueError("phase correlation: the volumes differ in shape")
    nz, ny, nx = fs.shape
    ws = _workspace(lib().aldvc_phase_correlation_workspace_size(nz, ny, nx))
    peak = torch.empty(1, dtype=torch.int64, device=fs.device)
    _lib.check(lib().aldvc_phase_correlation(_p(fs), _p(gs), nz, ny, nx, _p(peak), _p(ws), ws.numel(), stream_handle()),
               "aldvc_phase_correlation")
    i = int(peak.item())
    return i // (ny * nx), (i // nx) % ny, i % nx


# --------------------------------------------------------------------------- strain on the node grid
STRAIN_TYPES = {"infinitesimal": 0, "green_lagrange": 1, "euler_almansi": 2, "hencky": 3}


def _grid_args(grid_shape):
    nz, ny, nx = (int(s) for s in grid_shape)
    return nz, ny, nx


def gradient_plane_fit(U, grid_shape, spacing, halfwidth, valid=None):
    """(F (N, 3, 3), complete (N,) bool) of the FP64 (N, 3) field on the node grid (plane fit)."""
    U = dev(U, torch.float64).reshape(-1, 3).contiguous()
    N = U.shape[0]
    v = None if valid is None else dev(valid.to(torch.uint8) if isinstance(valid, torch.Tensor) else np.asarray(valid, np.uint8),
                                       torch.uint8).reshape(N)
    F = torch.empty((N, 3, 3), dtype=torch.float64, device=U.device)
    comp = torch.empty(N, dtype=torch.uint8, device=U.device)
    rx, ry, rz = (int(r) for r in halfwidth)
    hx, hy, hz = (float(h) for h in spacing)
    _lib.check(lib().aldvc_gradient_plane_fit(_p(U), _p(v), *_grid_args(grid_shape), hx, hy, hz, rx, ry, rz, _p(F), _p(comp),
                                              stream_handle()), "aldvc_gradient_plane_fit")
    return F, comp != 0


def gradient_fd(U, grid_shape, spacing, valid=None):
    """(F (N, 3, 3), complete (N,) bool) of the FP64 (N, 3) field by central / one-sided differences."""
    U = dev(U, torch.float64).reshape(-1, 3).contiguous()
    N = U.shape[0]
    v = None if valid is None else dev(valid.to(torch.uint8) if isinstance(valid, torch.Tensor) else np.asarray(valid, np.uint8),
                                       torch.uint8).reshape(N)
    F = torch.empty((N, 3, 3), dtype=torch.float64, device=U.device)
    comp = torch.empty(N, dtype=torch.uint8, device=U.device)
    hx, hy, hz = (float(h) for h in spacing)
    _lib.check(lib().aldvc_gradient_fd(_p(U), _p(v), *_grid_args(grid_shape), hx, hy, hz, _p(F), _p(comp), stream_handle()),
               "aldvc_gradient_fd")
    return F, comp != 0


def grid_smooth(field, grid_shape, sigma: float, valid=None) -> torch.Tensor:
    """Normalised Gaussian smoothing (sigma in nodes) of an FP64 grid field (N,); NaN / invalid nodes -> NaN."""
    x = dev(field, torch.float64).reshape(-1).contiguous()
    N = x.shape[0]
    v = None if valid is None else dev(valid.to(torch.uint8) if isinstance(valid, torch.Tensor) else np.asarray(valid, np.uint8),
                                       torch.uint8).reshape(N)
    w = gaussian_taps(sigma)
    if len(w) - 1 > 63:
        raise ValueError("grid_smooth: sigma too large (at most 63 taps each side)")
    out = torch.empty_like(x)
    nz, ny, nx = _grid_args(grid_shape)
    ws = _workspace(lib().aldvc_grid_smooth_workspace_size(nz, ny, nx))
    _lib.check(lib().aldvc_grid_smooth(_p(x), _p(v), nz, ny, nx, w.ctypes.data_as(ctypes.c_void_p), len(w) - 1, _p(out), _p(ws),
                                       ws.numel(), stream_handle()), "aldvc_grid_smooth")
    return out


def strain_measures(H, strain_type: str) -> dict:
    """Every strain measure of the physical gradients H (N, 3, 3): E, principal, max_shear, von_mises, volumetric,
    det_F, rotation_deg (FP64 CUDA tensors)."""
    H = dev(H, torch.float64).reshape(-1, 9).contiguous()
    N = H.shape[0]
    d = H.device
    out = {"E": torch.empty((N, 3, 3), dtype=torch.float64, device=d), "principal": torch.empty((N, 3), dtype=torch.float64, device=d)}
    for k in ("max_shear", "von_mises", "volumetric", "det_F", "rotation_deg"):
        out[k] = torch.empty(N, dtype=torch.float64, device=d)
    if strain_type not in STRAIN_TYPES:
        raise ValueError(f"unknown strain_type {strain_type!r}")
    _lib.check(lib().aldvc_strain_measures(_p(H), N, STRAIN_TYPES[strain_type], _p(out["E"]), _p(out["principal"]),
                                           _p(out["max_shear"]), _p(out["von_mises"]), _p(out["volumetric"]), _p(out["det_F"]),
                                           _p(out["rotation_deg"]), stream_handle()), "aldvc_strain_measures")
    return out


BOUNDARY_MIRROR, BOUNDARY_NEAREST = 0, 1
BSPLINE_HALF_TAPS = 32


def bspline_taps() -> np.ndarray:
    """Taps sqrt(3) z^j (j = 0..32, z = sqrt(3) - 2) of the cubic B-spline prefilter: the impulse response of the
    inverse of the sampling filter (z + 4 + 1/z) / 6; |z|^33 < 2e-19, so the tail is below FP64 resolution."""
    return np.sqrt(3.0) * (np.sqrt(3.0) - 2.0) ** np.arange(BSPLINE_HALF_TAPS + 1)


def gaussian_taps(sigma: float) -> np.ndarray:
    """Taps j = 0..r of the normalised Gaussian of scipy.ndimage.gaussian_filter (radius r = int(4 sigma + 0.5))."""
    r = int(4.0 * float(sigma) + 0.5)
    x = np.arange(-r, r + 1)
    phi = np.exp(-0.5 / (float(sigma) * float(sigma)) * x**2)
    phi = phi / phi.sum()
    return np.ascontiguousarray(phi[r:])


def sep_filter(vol: torch.Tensor, axis: int, taps, boundary: int, out: torch.Tensor | None = None) -> torch.Tensor:
    """One axis (0 = x, 1 = y, 2 = z) of the symmetric FIR ``aldvc_sep_filter`` over a float32 CUDA volume."""
    vol = dev(vol, torch.float32)
    w = np.ascontiguousarray(taps, dtype=np.float64)
    if len(w) - 1 > 63:
        raise ValueError("sep_filter: at most 63 taps each side (Gaussian sigma <= 15.6)")
    if out is None:
        out = torch.empty_like(vol)
    nz, ny, nx = vol.shape
    _lib.check(lib().aldvc_sep_filter(_p(vol), _p(out), nz, ny, nx, int(axis), w.ctypes.data_as(ctypes.c_void_p), len(w) - 1,
                                      int(boundary), stream_handle()), "aldvc_sep_filter")
    return out


def _three_axes(vol: torch.Tensor, taps, boundary: int) -> torch.Tensor:
    # axes z, y, x in turn, each rounded to float32: the order of scipy.ndimage's separable filters
    a = sep_filter(vol, 2, taps, boundary)
    b = sep_filter(a, 1, taps, boundary)
    return sep_filter(b, 0, taps, boundary, out=a)


def bspline_prefilter(vol: torch.Tensor) -> torch.Tensor:
    """Cubic B-spline coefficients of a float32 CUDA volume, mirror boundary (io/volume_ops.py:215-222)."""
    return _three_axes(vol, bspline_taps(), BOUNDARY_MIRROR)


def gaussian_presmooth(vol: torch.Tensor, sigma: float) -> torch.Tensor:
    """Gaussian smoothing with edge repeat (io/volume_ops.py:200-212); a float32 copy when sigma <= 0."""
    if sigma is None or sigma <= 0:
        return dev(vol, torch.float32).clone()
    return _three_axes(vol, gaussian_taps(sigma), BOUNDARY_NEAREST)


GRID_ODD_PAD = 10  # utils/grid_interp.py:40-45: odd reflection continues a node grid linearly past its edge (cubic only)
SPLINE_EDGE_PAD = 12  # SciPy's map_coordinates pads 'nearest' edges by 12 samples before its spline prefilter

_SPLINE_OPS: dict = {}


def spline_axis_operator(n: int) -> np.ndarray:
    """((n + pad) x n) FP64: along one axis of n nodes, the odd reflection by GRID_ODD_PAD (axes longer than one node),
    the edge padding by SPLINE_EDGE_PAD and the cubic B-spline prefilter of the edge-extended line (the 33-tap
    impulse response of bspline_taps, |z|^33 < 2e-19): the coefficients interp_grid_field's cubic interpolation
    evaluates, as one linear map of the axis's nodes.  Node 0 sits at coefficient index pad / 2."""
    if n not in _SPLINE_OPS:
        R = np.pad(np.eye(n), ((GRID_ODD_PAD, GRID_ODD_PAD), (0, 0)), mode="reflect", reflect_type="odd") if n > 1 else np.eye(n)
        E = np.concatenate([np.repeat(R[:1], SPLINE_EDGE_PAD, 0), R, np.repeat(R[-1:], SPLINE_EDGE_PAD, 0)])
        N = E.shape[0]
        taps = bspline_taps()
        J = len(taps) - 1
        rows = np.repeat(np.arange(N), 2 * J + 1)
        offs = np.tile(np.arange(-J, J + 1), N)
        S = np.zeros((N, N))
        np.add.at(S, (rows, np.clip(rows + offs, 0, N - 1)), taps[np.abs(offs)])
        _SPLINE_OPS[n] = np.ascontiguousarray(S @ E)
    return _SPLINE_OPS[n]


def grid_interp(field: torch.Tensor, grid_shape, origin, spacing, points: torch.Tensor, order: int = 3) -> torch.Tensor:
    """utils/grid_interp.py interp_grid_field on the device: the (N, C) or (N,) FP64 field of the node grid
    ``grid_shape`` (nz, ny, nx), node (iz, iy, ix) at ``origin`` + index * ``spacing`` ([x, y, z] each), sampled at
    ``points`` (M, 3) [x, y, z]; order 1 (trilinear) or 3 (cubic spline of the odd-reflected grid).  NaN nodes must
    be filled by the caller (the reference inpaints them first).  Returns (M, C) or (M,) FP64."""
    nz, ny, nx = (int(v) for v in grid_shape)
    f = dev(field, torch.float64)
    one = f.dim() == 1
    C = 1 if one else int(f.shape[1])
    pts = dev(points, torch.float64).reshape(-1, 3)
    M = pts.shape[0]
    out = torch.empty((M, C), dtype=torch.float64, device=f.device)
    ops = [None, None, None]
    pads = [0, 0, 0]
    ws = None
    if order == 3:
        for k, n in enumerate((nx, ny, nz)):
            op = spline_axis_operator(n)
            ops[k] = torch.from_numpy(op).to(f.device)
            pads[k] = op.shape[0] - n
        ws = _workspace(lib().aldvc_grid_interp_workspace_size(nz, ny, nx, C, *pads))
    ox, oy, oz = (float(v) for v in origin)
    hx, hy, hz = (float(v) for v in spacing)
    _lib.check(lib().aldvc_grid_interp(_p(f), nz, ny, nx, C, _p(ops[0]), _p(ops[1]), _p(ops[2]), pads[0], pads[1], pads[2], ox, oy, oz,
                                       hx, hy, hz, _p(pts), M, int(order), _p(out), _p(ws), 0 if ws is None else ws.numel(),
                                       stream_handle()), "aldvc_grid_interp")
    return out[:, 0] if one else out


def mask_fill(vol: torch.Tensor, mask: torch.Tensor, value: float) -> torch.Tensor:
    """In place: ``vol[mask == 0] = value`` (float32 volume, uint8/bool mask of the same shape)."""
    assert vol.is_cuda and vol.is_contiguous() and vol.dtype == torch.float32
    m = dev(mask.to(torch.uint8) if mask.dtype == torch.bool else mask, torch.uint8)
    if m.numel() != vol.numel():
        raise ValueError(f"mask_fill: mask shape {tuple(m.shape)} != volume shape {tuple(vol.shape)}")
    _lib.check(lib().aldvc_mask_fill(_p(vol), _p(m), vol.numel(), float(value), stream_handle()), "aldvc_mask_fill")
    return vol


def render_beads(accum: torch.Tensor, centres_zyx, peaks, sigma: float, radius: int) -> None:
    """Add Gaussian beads into an FP64 CUDA accumulator volume."""
    c = dev(centres_zyx, torch.float64).reshape(-1, 3)
    p = dev(peaks, torch.float64).reshape(-1)
    nz, ny, nx = accum.shape
    _lib.check(lib().aldvc_render_beads(_p(accum), nz, ny, nx, _p(c), _p(p), c.shape[0], float(sigma), int(radius),
                                        stream_handle()), "aldvc_render_beads")


def inpaint(values: torch.Tensor, grid_shape, unknown: torch.Tensor, tol: float = 1e-12, max_iter: int = 4000):
    """Fill the unknown nodes of an (N, C) FP64 field in place; returns (iters, err) device int32."""
    nz, ny, nx = (int(s) for s in grid_shape)
    C = 1 if values.dim() == 1 else int(values.shape[1])
    ws = _workspace(lib().aldvc_inpaint_workspace_size(nz, ny, nx, C))
    iters = torch.zeros(1, dtype=torch.int32, device=values.device)
    err = torch.zeros(1, dtype=torch.int32, device=values.device)
    _lib.check(lib().aldvc_inpaint(_p(values), nz, ny, nx, C, _p(unknown), float(tol), int(max_iter), _p(ws), ws.numel(), _p(iters),
                                   _p(err), stream_handle()), "aldvc_inpaint")
    return iters, err


def median_test(field: torch.Tensor, grid_shape, valid: torch.Tensor | None, threshold: float, eps: float = 0.1):
    """Universal median test of an (N, C) FP64 field; returns (flag uint8 (N,), err)."""
    nz, ny, nx = (int(s) for s in grid_shape)
    C = 1 if field.dim() == 1 else int(field.shape[1])
    flag = torch.empty(field.shape[0], dtype=torch.uint8, device=field.device)
    err = torch.zeros(1, dtype=torch.int32, device=field.device)
    ws = _workspace(lib().aldvc_median_test_workspace_size(nz, ny, nx, C))
    _lib.check(lib().aldvc_median_test(_p(field), nz, ny, nx, C, _p(valid), float(threshold), float(eps), _p(flag), _p(ws),
                                       ws.numel(), _p(err), stream_handle()), "aldvc_median_test")
    return flag, err
