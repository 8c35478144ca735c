"""Integer NCC search on the B200 (pyALDVC solver/integer_search.py:235-694).

``ncc_search``, ``ncc_search_expanding``, ``block_downsample``, ``phase_correlation_shift``,
``coarse_radius``, ``auto_pyramid_levels`` and ``pyramid_search`` keep the reference signatures and the
host contract (NumPy in, NumPy or a dict of NumPy arrays out).  Window placement, the ZNCC map, the
first-maximum argmax, PCE, the clipped flag and the 27-point sub-voxel fit all run in
``aldvc_ncc_search``; the integer peak is settled on FP64 re-scored values so it follows the reference's
FP64 map and tie rule.  The ``*_device`` forms take and return CUDA tensors (the pass's own path).
"""

from __future__ import annotations

import numpy as np

CLIPPED_EXPAND_FRACTION = 0.05  # integer_search.py:38
# integer_search.py:33-36, 563
PYRAMID_FINE_RADIUS = 2
COARSE_RADIUS_MARGIN = 1
MIN_COARSE_RADIUS = 2
MIN_PYRAMID_SUBSET = 8
MIN_COARSE_STD_RATIO = 0.35


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


# --------------------------------------------------------------------------- device forms
def _window_fits(shape, half, radius) -> bool:
    nz, ny, nx = (int(v) for v in shape)
    hx, hy, hz = (int(h) for h in half)
    rx, ry, rz = (int(r) for r in radius)
    return 2 * hx + 1 + 2 * rx <= nx and 2 * hy + 1 + 2 * ry <= ny and 2 * hz + 1 + 2 * rz <= nz


def ncc_search_expanding_device(f, g, coords, half, radius, shift0=None, auto_expand: bool = True, max_expand: int = 3,
                                engine_of=None, calls: list | None = None, search_fn=None) -> dict:
    """Device ``ncc_search_expanding`` (integer_search.py:486-524) on CUDA tensors: ``coords`` (N,3) int64, ``half``
    the template half-widths, ``shift0`` (N,3) int64 or None.  Returns disp, cc, pce (FP64), clipped, ok (bool)
    tensors, the final ``radius`` and the number of ``expansions``.  ``engine_of(half, radius)`` picks the NCC
    engine of each search (tiled by default); ``calls`` collects (nodes, half, radius, engine) per search.
    ``search_fn(coords, half, radius, shift, engine)`` replaces the search over whole device volumes (the tiled
    pass runs it box by box from host memory); ``f`` then only has to give the volume's ``shape``."""
    import torch

    K = _kernels()
    N = int(coords.shape[0])
    rad = tuple(int(r) for r in radius)
    dev = coords.device
    out = {"disp": torch.full((N, 3), float("nan"), dtype=torch.float64, device=dev),
           "cc": torch.full((N,), float("nan"), dtype=torch.float64, device=dev),
           "pce": torch.full((N,), float("nan"), dtype=torch.float64, device=dev),
           "clipped": torch.zeros(N, dtype=torch.bool, device=dev), "ok": torch.zeros(N, dtype=torch.bool, device=dev),
           "radius": rad, "expansions": 0}
    if N == 0 or not _window_fits(f.shape, half, rad):
        return out

    def search(c, r, sh):
        eng = K.NCC_TILED if engine_of is None else engine_of(half, r)
        if calls is not None:
            calls.append((int(c.shape[0]), tuple(half), tuple(r), eng))
        res = K.ncc_search(f, g, c, half, r, sh, eng) if search_fn is None else search_fn(c, half, r, sh, eng)
        return {"disp": res["disp"], "cc": res["cc"], "pce": res["pce"], "clipped": res["clipped"] != 0, "ok": res["ok"] != 0}

    out.update(search(coords, rad, shift0))
    for _ in range(max_expand if auto_expand else 0):
        sel = out["clipped"] & out["ok"]
        n_ok = int(out["ok"].sum().item())
        n_sel = int(sel.sum().item())
        if n_ok == 0 or n_sel <= CLIPPED_EXPAND_FRACTION * n_ok:
            break
        rad = tuple(2 * r for r in rad)
        if not _window_fits(f.shape, half, rad):
            break  # the window no longer fits in the volume: keep the previous peaks
        idx = torch.nonzero(sel).flatten()
        sub = search(coords[idx].contiguous(), rad, None if shift0 is None else shift0[idx].contiguous())
        s_ok = sub["ok"]
        if not bool(s_ok.any().item()):
            break
        take = idx[s_ok]
        for key in ("disp", "cc", "pce", "clipped", "ok"):
            out[key][take] = sub[key][s_ok]
        out["expansions"] += 1
        out["radius"] = rad
    return out


def clean_field_device(disp, grid_shape, threshold: float, errs=None):
    """``_clean_field`` (integer_search.py:545-555) on the device: median-test outliers and non-finite rows of the
    (N,3) FP64 field are replaced by the spring inpainting of their neighbours (every row bad -> zeros).  The
    device error words go to ``errs`` (a kernels.ErrorWords), else they are checked here."""
    import torch

    K = _kernels()
    own = errs is None
    errs = K.ErrorWords() if own else errs
    d = disp.clone()
    good = torch.isfinite(d).all(dim=1)
    if threshold > 0 and int(good.sum().item()) > 27:
        flag, e = K.median_test(torch.where(good[:, None], d, torch.nan).contiguous(), grid_shape,
                                good.to(torch.uint8).contiguous(), threshold)
        errs.add(e, "median_test")
        good = good & (flag == 0)
    bad = ~good
    if bool(bad.all().item()):
        return torch.zeros_like(d)
    d[bad] = 0.0
    d = d.contiguous()
    _, e = K.inpaint(d, grid_shape, bad.to(torch.uint8).contiguous())
    errs.add(e, "inpaint")
    if own:
        errs.check()
    return d


def coarse_radius(radius, fac: int) -> tuple:
    """Search radius at a coarse level (integer_search.py:566-572): ceil(radius / fac) + 1, at least 2."""
    return tuple(max(MIN_COARSE_RADIUS, -(-int(r) // fac) + COARSE_RADIUS_MARGIN) for r in radius)


def _device_volume(v):
    import torch

    K = _kernels()
    if isinstance(v, torch.Tensor):
        return K.dev(v, torch.float32), True
    return K.dev(np.ascontiguousarray(np.asarray(v, dtype=np.float32)), torch.float32), False


def block_downsample(vol, factor: int):
    """Block-mean downsampling by an integer ``factor``, trailing voxels dropped (integer_search.py:235-244);
    FP64 block sums, float32 result."""
    K = _kernels()
    v, keep = _device_volume(vol)
    out = K.block_downsample(v, int(factor))
    return out if keep else out.cpu().numpy()


def phase_correlation_shift_device(f, g, voi=None, max_dim: int = 128, downsample=None) -> np.ndarray:
    """Global integer shift (dx, dy, dz) of ``g`` against ``f`` (integer_search.py:247-291): the VOI block-
    downsampled until no axis exceeds ``max_dim``, Hann-windowed phase correlation, peak wrapped and scaled.
    ``downsample(factor)`` gives the block-mean pair of a volume that is not on the device (``f`` then only gives
    the shape; no VOI)."""
    import math

    K = _kernels()
    if voi is not None:
        sl = voi.clamp(tuple(f.shape)).slices
        f = f[sl].contiguous()
        g = g[sl].contiguous()
    factor = max(1, int(math.ceil(max(f.shape) / max_dim)))
    if downsample is not None and factor > 1:
        fs, gs = downsample(factor)
    else:
        fs = K.block_downsample(f, factor)
        gs = K.block_downsample(g, factor)
    peak = np.array(K.phase_correlation_peak(fs, gs), dtype=np.float64)
    for ax, n in enumerate(fs.shape):
        if peak[ax] > n // 2:
            peak[ax] -= n
    dz, dy, dx = peak * factor
    return np.array([dx, dy, dz], dtype=np.float64)


def phase_correlation_shift(f, g, voi=None, max_dim: int = 128) -> np.ndarray:
    fd, _ = _device_volume(f)
    gd, _ = _device_volume(g)
    return phase_correlation_shift_device(fd, gd, voi, max_dim)


phase_correlation_shift.__doc__ = phase_correlation_shift_device.__doc__


def auto_pyramid_levels(shape, subset, radius, max_levels: int = 3, f=None, min_std_ratio: float = MIN_COARSE_STD_RATIO,
                        std0: float | None = None, downsample=None) -> int:
    """Coarse levels that fit the search window and keep the texture (integer_search.py:575-612): level l
    (factor 2^l) is taken while every axis holds the level's window plus margin and, with ``f``, the block-mean
    volume keeps at least ``min_std_ratio`` of the full-resolution standard deviation.  A volume that is not on
    the device gives its standard deviation ``std0`` and ``downsample(factor)`` (its block means, on the device)
    instead of ``f``."""
    K = _kernels()
    fd = None if f is None else _device_volume(f)[0]
    if fd is not None:
        std0 = float(K.volume_stats(fd)[1].item())
        downsample = lambda fac: K.block_downsample(fd, fac)  # noqa: E731
    levels = 0
    for lv in range(1, max_levels + 1):
        fac = 2**lv
        fits = True
        for n, w, r in zip(tuple(shape)[::-1], subset, coarse_radius(radius, fac)):
            w_l = max(MIN_PYRAMID_SUBSET, (int(w) // fac) // 2 * 2)
            if int(n) // fac < w_l + 1 + 2 * max(r, 1) + 4:
                fits = False
        if fits and std0 is not None and std0 > 0:
            ds = downsample(fac)
            if float(K.volume_stats(ds)[1].item()) < min_std_ratio * std0:
                fits = False
        if fits:
            levels = lv
        else:
            break
    return levels


def pyramid_search_device(f, g, coords, grid_shape, subset, radius, levels: int = 0, global_shift=None,
                          outlier_threshold: float = 2.0, auto_expand: bool = True, max_expand: int = 3,
                          fine_radius: int = PYRAMID_FINE_RADIUS, valid=None, engine_of=None, calls: list | None = None,
                          errs=None, level_volumes=None, search_fn=None) -> dict:
    """Coarse-to-fine NCC search (integer_search.py:615-694) on CUDA tensors: the coarsest level searches
    ``coarse_radius(radius)`` on block means, each finer level refines with ``fine_radius`` around the up-scaled,
    median-cleaned and inpainted estimate.  ``valid`` (N,) bool restricts the searched nodes.  Returns disp (N,3)
    FP64 in full-resolution voxels, the last level's ok / cc / pce / clipped, and the per-level record.  The
    cleaning's device error words go to ``errs`` (a kernels.ErrorWords), else they are checked per level.
    A pass over volumes streamed from host memory gives ``level_volumes(factor)`` (the block-mean pair of a
    coarse level, on the device), ``search_fn`` (the full-resolution search, see ncc_search_expanding_device)
    and a resolved ``levels`` (0: the full-resolution search alone); ``f`` and ``g`` then only give the volume shape."""
    import torch

    K = _kernels()
    streamed = level_volumes is not None
    if level_volumes is None:
        level_volumes = lambda fac: (K.block_downsample(f, fac), K.block_downsample(g, fac))  # noqa: E731
    if levels <= 0 and not streamed:
        levels = auto_pyramid_levels(tuple(f.shape), subset, radius, f=f)
    N = int(coords.shape[0])
    active = torch.arange(N, device=coords.device) if valid is None else torch.nonzero(valid).flatten()
    if active.numel() == 0:
        active = torch.arange(N, device=coords.device)
    disp_full = torch.zeros((N, 3), dtype=torch.float64, device=coords.device)
    if global_shift is not None:
        disp_full += torch.as_tensor(np.asarray(global_shift, dtype=np.float64), device=coords.device)[None, :]
    info: dict = {"levels": levels, "per_level": [], "expansions": 0, "n_searched": int(active.numel())}
    for lv in range(levels, -1, -1):
        fac = 2**lv
        fl, gl = level_volumes(fac) if fac > 1 else (f, g)
        subset_l = tuple(max(MIN_PYRAMID_SUBSET, (int(w) // fac) // 2 * 2) for w in subset)
        half_l = tuple(w // 2 for w in subset_l)
        rad_l = coarse_radius(radius, fac) if lv == levels else (int(fine_radius),) * 3
        coords_l = torch.round(coords[active].double() / fac).long().contiguous()
        shift_l = torch.round(disp_full[active] / fac).long().contiguous()
        sub = ncc_search_expanding_device(fl, gl, coords_l, half_l, rad_l, shift_l, auto_expand, max_expand, engine_of, calls,
                                          search_fn if fac == 1 else None)
        res = {k: sub[k] for k in ("radius", "expansions")}
        for key, fill in (("disp", float("nan")), ("cc", float("nan")), ("pce", float("nan"))):
            t = torch.full((N,) + tuple(sub[key].shape[1:]), fill, dtype=torch.float64, device=coords.device)
            t[active] = sub[key]
            res[key] = t
        for key in ("clipped", "ok"):
            t = torch.zeros(N, dtype=torch.bool, device=coords.device)
            t[active] = sub[key]
            res[key] = t
        info["expansions"] += res["expansions"]
        d = res["disp"] * fac
        d[~res["ok"]] = float("nan")
        n_ok = int(res["ok"].sum().item())
        rec = {"level": lv, "n_ok": n_ok, "radius": res["radius"], "subset": subset_l}
        if n_ok == 0:
            info["per_level"].append(rec)
            continue
        disp_full = clean_field_device(d, grid_shape, outlier_threshold, errs)
        rec["median_cc"] = float(np.nanmedian(res["cc"].cpu().numpy()))
        rec["clipped_frac"] = float(res["clipped"][res["ok"]].double().mean().item())
        info["per_level"].append(rec)
        for key in ("cc", "pce", "ok", "clipped"):
            info[key] = res[key]
    info["disp"] = disp_full
    return info


def pyramid_search(f, g, coords, grid_shape, subset, radius, levels: int = 0, global_shift=None, outlier_threshold: float = 2.0,
                   auto_expand: bool = True, max_expand: int = 3, fine_radius: int = PYRAMID_FINE_RADIUS, backend: str = "cuda",
                   valid=None) -> dict:
    """Host contract of ``pyramid_search_device`` (integer_search.py:615-694): NumPy in, NumPy arrays out;
    ``backend`` is accepted for signature compatibility (the search runs on the device)."""
    import torch

    fd, _ = _device_volume(f)
    gd, _ = _device_volume(g)
    c = torch.from_numpy(np.ascontiguousarray(np.asarray(coords, dtype=np.int64))).cuda()
    v = None if valid is None else torch.from_numpy(np.ascontiguousarray(np.asarray(valid, dtype=bool))).cuda()
    info = pyramid_search_device(fd, gd, c, tuple(int(n) for n in grid_shape), subset, radius, levels, global_shift,
                                 outlier_threshold, auto_expand, max_expand, fine_radius, v)
    return {k: (v_.cpu().numpy() if isinstance(v_, torch.Tensor) else v_) for k, v_ in info.items()}
