"""Drop-in for ``al_dvc.solver.cuda_kernels`` (pyALDVC v1.2.1, solver/cuda_kernels.py:107-1755).

Same function names, arguments and host contract as the reference module:

* inputs are host NumPy arrays; outputs are fresh host arrays; ``P0`` / ``U_old`` are never mutated;
  ``zncc_direct_cuda`` fills the caller's ``out`` (cuda_kernels.py:1397-1755);
* the ``(1, 1, 1)`` gradient placeholders select the on-the-fly stencil and the ``(1, 1, 1)`` mask
  placeholder means "no mask" (numba_kernels.py:188-212, 314-317);
* volumes are uploaded once per host array object and cached (LRU of 8, cuda_kernels.py:184-214);
* numerical failures are per-node status codes, never exceptions.

The work itself is the B200 library (``include/aldvc_b200.h``).  There is no CPU fallback: every
function raises when the CUDA library or a device is unusable.  The reference module's names
``cuda_available``, ``unavailable_reason``, ``unavailable_kind``, ``device_name`` and
``clear_device_cache`` are kept so the reference's backend switch (local_icgn.resolve_backend
:110-123) can route its own pipeline through this module.
"""

from __future__ import annotations

import threading
from collections import OrderedDict

import numpy as np

STATUS_INVALID_SUBSET = 3
STATUS_SKIPPED = 6
CHUNK_NODES = 1 << 30  # one persistent launch per call unless the caller asks for chunks
TPL_MAX = 35937  # largest NCC template held in shared memory (33^3 voxels)
DEVICE_CACHE_SIZE = 8

_available: bool | None = None
_unavailable_reason = ""
_unavailable_kind = ""
_probe_lock = threading.Lock()


# --------------------------------------------------------------------------- availability (cuda_kernels.py:107-180)
def cuda_available() -> bool:
    global _available
    if _available is not None:
        return _available
    with _probe_lock:
        if _available is not None:
            return _available
        return _probe_once()


def _probe_once() -> bool:
    global _available, _unavailable_reason, _unavailable_kind
    kind = "missing"
    try:
        import torch

        from . import _lib

        _lib.load()
        kind = "no_device"
        if not torch.cuda.is_available():
            raise RuntimeError("torch reports no usable CUDA device")
        kind = "error"
        major, minor = torch.cuda.get_device_capability()
        if (major, minor) != (10, 0):
            raise RuntimeError(f"the library is built for sm_100a, device is sm_{major}{minor}")
        _available, _unavailable_kind = True, ""
    except Exception as exc:  # missing library, no device, wrong architecture
        _unavailable_reason = f"{type(exc).__name__}: {exc}"
        _unavailable_kind = kind
        _available = False
    return _available


def unavailable_reason() -> str:
    cuda_available()
    return _unavailable_reason


def unavailable_kind() -> str:
    cuda_available()
    return _unavailable_kind


def device_name() -> str:
    if not cuda_available():
        return ""
    import torch

    return torch.cuda.get_device_name()


def _require():
    if not cuda_available():
        raise RuntimeError(f"pyaldvc_b200 CUDA backend unavailable ({_unavailable_reason})")
    from . import kernels

    return kernels


# --------------------------------------------------------------------------- device cache (cuda_kernels.py:184-214)
class DeviceCache:
    """Host array -> device tensor, keyed by the host object; bounded LRU."""

    def __init__(self, size: int = DEVICE_CACHE_SIZE) -> None:
        self._items: OrderedDict[tuple, tuple] = OrderedDict()
        self._size = size

    def get(self, arr: np.ndarray, dtype):
        import torch

        key = (id(arr), arr.shape, str(arr.dtype), str(dtype))
        hit = self._items.get(key)
        if hit is not None and hit[0] is arr:
            self._items.move_to_end(key)
            return hit[1]
        t = torch.from_numpy(np.ascontiguousarray(arr)).to(device="cuda", dtype=dtype)
        self._items[key] = (arr, t)  # keep the host array alive so its id stays unique
        while len(self._items) > self._size:
            self._items.popitem(last=False)
        return t

    def get_quads(self, arr: np.ndarray):
        """The overlapping-quad copy of ``arr`` (16 bytes per voxel, ``kernels.make_quads``), cached like ``get``."""
        key = (id(arr), arr.shape, str(arr.dtype), "quads")
        hit = self._items.get(key)
        if hit is not None and hit[0] is arr:
            self._items.move_to_end(key)
            return hit[1]
        import torch

        from . import kernels

        q = kernels.make_quads(self.get(arr, torch.float32))
        self._items[key] = (arr, q)
        while len(self._items) > self._size:
            self._items.popitem(last=False)
        return q

    def clear(self) -> None:
        self._items.clear()


_cache = DeviceCache()


def clear_device_cache() -> None:
    _cache.clear()


def _volumes(f, gx, gy, gz, mask, g=None):
    """Device tensors with the reference's placeholder conventions resolved to NULL pointers."""
    import torch

    f_d = _cache.get(f, torch.float32)
    stored = np.shape(gx) == np.shape(f)
    gx_d = _cache.get(gx, torch.float32) if stored else None
    gy_d = _cache.get(gy, torch.float32) if stored else None
    gz_d = _cache.get(gz, torch.float32) if stored else None
    m_d = _cache.get(mask, torch.uint8) if np.shape(mask) == np.shape(f) else None
    g_d = None if g is None else _cache.get(g, torch.float32)
    return f_d, gx_d, gy_d, gz_d, m_d, g_d


def _split(split_index, split_keep):
    import torch

    if split_index is None or split_keep is None:
        return None, None
    return (torch.from_numpy(np.ascontiguousarray(split_index, dtype=np.int64)).cuda(),
            torch.from_numpy(np.ascontiguousarray(split_keep, dtype=np.uint8)).cuda())


def _chunks(n: int, chunk: int):
    chunk = max(1, int(chunk))
    for start in range(0, n, chunk):
        yield start, min(n, start + chunk)


def _tensor_grid(coords):
    """(xs, ys, zs) when the (N, 3) [x, y, z] node coordinates are the tensor grid of those axes in mesh order (x
    fastest, then y, then z), else None."""
    c = np.asarray(coords)
    if c.ndim != 2 or c.shape[1] != 3 or c.shape[0] == 0:
        return None
    xs, ys, zs = (np.unique(c[:, k]) for k in range(3))
    if len(xs) * len(ys) * len(zs) != c.shape[0]:
        return None
    Z, Y, X = np.meshgrid(zs, ys, xs, indexing="ij")
    if not (np.array_equal(c[:, 0], X.ravel()) and np.array_equal(c[:, 1], Y.ravel()) and np.array_equal(c[:, 2], Z.ravel())):
        return None
    return tuple(np.ascontiguousarray(a, dtype=np.int64) for a in (xs, ys, zs))


# --------------------------------------------------------------------------- kernels
def precompute_nodes_cuda(coords, hx, hy, hz, f, gx, gy, gz, mask, min_valid_ratio, cond_max, stride=1, split_index=None,
                          split_keep=None, chunk: int = CHUNK_NODES):
    """Same contract as ``numba_kernels.precompute_nodes`` (:499-509), on the B200.  Nodes that form a tensor grid (a
    mesh) with stored gradients, stride 1 and no split rows take the separable form (``aldvc_precompute_grid``)."""
    K = _require()
    vols = _volumes(f, gx, gy, gz, mask)
    si, sk = _split(split_index, split_keep)
    axes = _tensor_grid(coords) if (si is None and int(stride) == 1 and vols[1] is not None and np.shape(f)[2] <= 8192) else None
    if axes is not None:  # the nodes of a tensor grid (a mesh): separable moment sums
        H, L, mf, bf, nv, valid = K.precompute_grid(*axes, (hx, hy, hz), vols[0], vols[1], vols[2], vols[3], min_valid_ratio,
                                                    cond_max, vols[4])
    else:
        H, L, mf, bf, nv, valid = K.precompute(coords, (hx, hy, hz), *vols[:5], min_valid_ratio, cond_max, stride, si, sk)
    return (H.cpu().numpy(), L.cpu().numpy(), mf.cpu().numpy(), bf.cpu().numpy(), nv.cpu().numpy(),
            valid.cpu().numpy().astype(bool))


def icgn_12dof_cuda(coords, P0, hx, hy, hz, f, gx, gy, gz, mask, g, mode, L_all, meanf_all, bottomf_all, valid, tol, dp_tol,
                    max_iter, patience, stride=1, H_all=None, pattern=None, noise_gain=0.0, predictive=True, split_index=None,
                    split_keep=None, chunk: int = CHUNK_NODES, progress_fn=None, variant: int = 0, threads: int = 0,
                    brick_floats: int = 0):
    """Same contract as ``numba_kernels.icgn_12dof_parallel`` (:1211-1278), on the B200.

    ``chunk`` nodes per launch (default: all in one persistent launch); ``progress_fn(fraction)``
    after each.  ``variant`` 0 = batched persistent kernel, 1 = plain one-node-per-block kernel.
    """
    import torch

    K = _require()
    N = int(np.asarray(coords).shape[0])
    P_out = np.array(P0, dtype=np.float64).reshape(N, 12).copy()
    n_iter = np.zeros(N, dtype=np.int32)
    status = np.full(N, STATUS_SKIPPED, dtype=np.int8)
    zncc = np.full(N, np.nan)
    if N == 0:
        return P_out, n_iter, status, zncc
    f_d, gx_d, gy_d, gz_d, m_d, g_d = _volumes(f, gx, gy, gz, mask, g)
    coords_d = torch.from_numpy(np.ascontiguousarray(coords, dtype=np.int64)).cuda()
    P0_d = torch.from_numpy(P_out).cuda()
    L_d = torch.from_numpy(np.ascontiguousarray(L_all, dtype=np.float64)).cuda()
    mf_d = torch.from_numpy(np.ascontiguousarray(meanf_all, dtype=np.float64)).cuda()
    v_d = torch.from_numpy(np.ascontiguousarray(valid, dtype=np.uint8)).cuda()
    use_noise = H_all is not None and pattern is not None and noise_gain > 0.0
    H_d = torch.from_numpy(np.ascontiguousarray(H_all, dtype=np.float64)).cuda() if use_noise else None
    pat = np.ascontiguousarray(pattern, dtype=np.float64) if use_noise else None
    si, sk = _split(split_index, split_keep)
    g4 = _cache.get_quads(g) if (mode != 0 and variant == K.BATCHED) else None
    for start, stop in _chunks(N, chunk):
        sl = slice(start, stop)
        si_c = None if si is None else si[sl]
        P, it, st, zc = K.icgn12(coords_d[sl], P0_d[sl], (hx, hy, hz), f_d, gx_d, gy_d, gz_d, m_d, g_d, mode, L_d[sl], mf_d[sl],
                                 v_d[sl], tol, dp_tol, max_iter, patience, stride, None if H_d is None else H_d[sl], pat,
                                 noise_gain if use_noise else 0.0, predictive, si_c, sk, variant, threads, brick_floats, g4=g4)
        P_out[sl] = P.cpu().numpy()
        n_iter[sl] = it.cpu().numpy()
        status[sl] = st.cpu().numpy()
        zncc[sl] = zc.cpu().numpy()
        if progress_fn is not None:
            progress_fn(min(1.0, stop / N))
    return P_out, n_iter, status, zncc


def icgn_3dof_cuda(coords, U_old, F_fixed, vdual, hx, hy, hz, f, gx, gy, gz, mask, g, mode, H_all, meanf_all, bottomf_all, valid,
                   mu, tol, dp_tol, max_iter, patience, stride=1, n_full=0.0, noise_gain=0.0, predictive=True, split_index=None,
                   split_keep=None, chunk: int = CHUNK_NODES, progress_fn=None, variant: int = 0, threads: int = 0,
                   brick_floats: int = 0):
    """Same contract as ``numba_kernels.icgn_3dof_parallel`` (:1281-1346), on the B200."""
    import torch

    K = _require()
    N = int(np.asarray(coords).shape[0])
    U_out = np.array(U_old, dtype=np.float64).reshape(N, 3).copy()
    n_iter = np.zeros(N, dtype=np.int32)
    status = np.full(N, STATUS_SKIPPED, dtype=np.int8)
    zncc = np.full(N, np.nan)
    if N == 0:
        return U_out, n_iter, status, zncc
    f_d, gx_d, gy_d, gz_d, m_d, g_d = _volumes(f, gx, gy, gz, mask, g)

    def up(a, shape):
        return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64).reshape(shape)).cuda()

    coords_d = torch.from_numpy(np.ascontiguousarray(coords, dtype=np.int64)).cuda()
    U_d, F_d, vd_d = up(U_out, (N, 3)), up(F_fixed, (N, 9)), up(vdual, (N, 3))
    H_d = up(H_all, (N, 12, 12))
    mf_d, bf_d = up(meanf_all, (N,)), up(bottomf_all, (N,))
    v_d = torch.from_numpy(np.ascontiguousarray(valid, dtype=np.uint8)).cuda()
    si, sk = _split(split_index, split_keep)
    g4 = _cache.get_quads(g) if (mode != 0 and variant == K.BATCHED) else None
    for start, stop in _chunks(N, chunk):
        sl = slice(start, stop)
        U, it, st, zc = K.icgn3(coords_d[sl], U_d[sl], F_d[sl], vd_d[sl], (hx, hy, hz), f_d, gx_d, gy_d, gz_d, m_d, g_d, mode,
                                H_d[sl], mf_d[sl], bf_d[sl], v_d[sl], mu, tol, dp_tol, max_iter, patience, stride, n_full,
                                noise_gain if noise_gain > 0.0 else 0.0, predictive, None if si is None else si[sl], sk, variant,
                                threads, brick_floats, g4=g4)
        U_out[sl] = U.cpu().numpy()
        n_iter[sl] = it.cpu().numpy()
        status[sl] = st.cpu().numpy()
        zncc[sl] = zc.cpu().numpy()
        if progress_fn is not None:
            progress_fn(min(1.0, stop / N))
    return U_out, n_iter, status, zncc


def zncc_direct_cuda(f, g, coords, hx, hy, hz, rx, ry, rz, wx0, wy0, wz0, t_ok, out) -> None:
    """Same contract as ``integer_search._zncc_direct`` (:44-151): fills ``out`` in place, on the B200."""
    import torch

    K = _require()
    n = int(np.asarray(coords).shape[0])
    if n == 0:
        return
    f_d = _cache.get(f, torch.float32)
    g_d = _cache.get(g, torch.float32)
    m = K.ncc_map(f_d, g_d, np.ascontiguousarray(coords, dtype=np.int64), (hx, hy, hz), (rx, ry, rz), wx0, wy0, wz0,
                  np.asarray(t_ok, dtype=np.uint8))
    out[...] = m.cpu().numpy()
