"""Integer NCC search on the B200 (pyALDVC solver/integer_search.py:329-524).

``ncc_search`` and ``ncc_search_expanding`` keep the reference signatures and the host contract
(NumPy in, dict of NumPy arrays out).  Window placement, the ZNCC map, the first-maximum argmax,
PCE, the clipped flag and the 27-point sub-voxel fit all run in ``aldvc_ncc_search``; the integer
peak is settled on FP64 re-scored values so it follows the reference's FP64 map and tie rule.
"""

from __future__ import annotations

import numpy as np

CLIPPED_EXPAND_FRACTION = 0.05  # integer_search.py:38


def _kernels():
    from .cuda_kernels import _require

    return _require()


def ncc_search_device(f_d, g_d, coords, subset, radius, shift0=None) -> dict:
    """Device-tensor search: ``f_d``/``g_d`` CUDA float32 volumes; returns a dict of CUDA tensors."""
    K = _kernels()
    half = tuple(int(w) // 2 for w in subset)
    return K.ncc_search(f_d, g_d, coords, half, radius, shift0)


def ncc_search(f, g, coords, subset, radius, shift0=None, chunk: int = 64, backend: str = "cuda", engine: int = 0) -> dict:
    """Per-node NCC search (integer_search.ncc_search :329-483); ``chunk`` and ``backend`` are accepted for
    signature compatibility, the device chunks by its workspace.  ``engine`` 0 = tiled, 1 = plain."""
    import torch

    from .cuda_kernels import _cache

    K = _kernels()
    f = np.asarray(f, dtype=np.float32)
    g = np.asarray(g, dtype=np.float32)
    nz, ny, nx = f.shape
    coords = np.asarray(coords, dtype=np.int64)
    N = coords.shape[0]
    hx, hy, hz = (int(w) // 2 for w in subset)
    rx, ry, rz = (int(r) for r in radius)
    wx, wy, wz = 2 * hx + 1 + 2 * rx, 2 * hy + 1 + 2 * ry, 2 * hz + 1 + 2 * rz
    out = {"disp": np.full((N, 3), np.nan), "cc": np.full(N, np.nan), "pce": np.full(N, np.nan),
           "clipped": np.zeros(N, dtype=bool), "ok": np.zeros(N, dtype=bool)}
    if N == 0 or wx > nx or wy > ny or wz > nz:
        return out
    sh = None if shift0 is None else np.asarray(np.round(shift0), dtype=np.int64).reshape(N, 3)
    f_d = _cache.get(f, torch.float32)
    g_d = _cache.get(g, torch.float32)
    res = K.ncc_search(f_d, g_d, coords, (hx, hy, hz), (rx, ry, rz), sh, engine)
    out["disp"] = res["disp"].cpu().numpy()
    out["cc"] = res["cc"].cpu().numpy()
    out["pce"] = res["pce"].cpu().numpy()
    out["clipped"] = res["clipped"].cpu().numpy().astype(bool)
    out["ok"] = res["ok"].cpu().numpy().astype(bool)
    return out


def ncc_search_expanding(f, g, coords, subset, radius, shift0=None, auto_expand: bool = True, max_expand: int = 3,
                         chunk: int = 64, backend: str = "cuda", engine: int = 0) -> dict:
    """``ncc_search`` plus radius doubling for clipped peaks (integer_search.ncc_search_expanding :486-524)."""
    res = ncc_search(f, g, coords, subset, radius, shift0, engine=engine)
    res["expansions"] = 0
    res["radius"] = tuple(int(r) for r in radius)
    rad = res["radius"]
    for _ in range(max_expand if auto_expand else 0):
        sel = res["clipped"] & res["ok"]
        n_ok = int(res["ok"].sum())
        if n_ok == 0 or sel.sum() <= CLIPPED_EXPAND_FRACTION * n_ok:
            break
        rad = tuple(2 * r for r in rad)
        sub_shift = None if shift0 is None else np.asarray(shift0)[sel]
        sub = ncc_search(f, g, np.asarray(coords)[sel], subset, rad, sub_shift, engine=engine)
        if not sub["ok"].any():
            break
        idx = np.flatnonzero(sel)[sub["ok"]]
        for key in ("disp", "cc", "pce", "clipped", "ok"):
            res[key][idx] = sub[key][sub["ok"]]
        res["expansions"] += 1
        res["radius"] = rad
    return res
