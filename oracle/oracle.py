"""CPU oracle for the AL-DVC hot path (test infrastructure only).

This module is the checker: only ``tests/``, ``__graft_entry__.smoke()`` and
``bench.py``'s CPU-baseline leg import it.  The product package
``pyaldvc_b200`` never imports, links or calls anything under ``oracle/``.

The per-node kernels are a plain-C FP64 restatement (``aldvc_oracle.c``) of
pyALDVC's Numba CPU kernels; the orchestration around them is restated here
in NumPy/SciPy.  Every function cites the reference file:line it follows
(paths inside the pyALDVC project, ``src/al_dvc/...``).  Parity with the
reference is pinned by ``tests/golden/*.npz`` (made by
``tests/golden/make_golden.py``, which imports the reference).
"""

from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np
from scipy import sparse

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liborc_aldvc.so")
_lib = None

STATUS_CONVERGED, STATUS_MAX_ITER, STATUS_OUT_OF_BOUNDS, STATUS_INVALID_SUBSET = 0, 1, 2, 3
STATUS_SINGULAR, STATUS_NAN, STATUS_SKIPPED, STATUS_STALLED = 4, 5, 6, 7

_P = ctypes.c_void_p
_I64 = ctypes.c_int64
_I = ctypes.c_int
_D = ctypes.c_double


def build() -> str:
    """Compile the C oracle with its Makefile (idempotent)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        L.orc_num_threads.restype = _I
        L.orc_set_num_threads.argtypes = [_I]
        L.orc_sample_points.argtypes = [_P, _I64, _I64, _I64, _P, _P, _P, _I64, _I, _P]
        L.orc_gradients.argtypes = [_P, _I64, _I64, _I64, _I64, _P, _P, _P]
        L.orc_compose_warp.argtypes = [_P, _P]
        L.orc_compose_warp.restype = _I
        L.orc_precompute.argtypes = [_P, _I64, _I, _I, _I, _I, _P, _P, _P, _P, _I, _P, _I64, _I64, _I64, _P, _P, _I64, _D, _D,
                                     _P, _P, _P, _P, _P, _P]
        L.orc_icgn12.argtypes = [_P, _I64, _P, _I, _I, _I, _I, _P, _P, _P, _P, _I, _P, _P, _I64, _I64, _I64, _I, _P, _P, _D, _D, _I,
                                 _I, _P, _P, _D, _I, _P, _P, _I64, _P, _P, _P, _P]
        L.orc_icgn3.argtypes = [_P, _I64, _P, _P, _P, _I, _I, _I, _I, _P, _P, _P, _P, _I, _P, _P, _I64, _I64, _I64, _I, _P, _P, _P,
                                _D, _D, _D, _I, _I, _D, _D, _I, _P, _P, _I64, _P, _P, _P, _P]
        L.orc_zncc_direct.argtypes = [_P, _P, _I64, _I64, _I64, _P, _I64, _I, _I, _I, _I, _I, _I, _P, _P, _P, _P, _P]
        L.orc_znssd.argtypes = [_P, _P, _I64, _I64, _I64, _P, _I64, _I, _I, _I, _I, _P, _P]
        L.orc_sep_filter.argtypes = [_P, _P, _I64, _I64, _I64, _I, _P, _I, _I]
        L.orc_window_box_stats.argtypes = [_P, _I64, _I64, _I64, _I64, _I64, _I64, _I64, _P, _P]
        _lib = L
    return _lib


def num_threads() -> int:
    return int(lib().orc_num_threads())


def set_num_threads(n: int) -> None:
    lib().orc_set_num_threads(int(n))


def _ptr(a):
    return None if a is None else a.ctypes.data


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def _vol_args(f, gx, gy, gz, mask):
    """Placeholders follow the reference: (1,1,1) gradients = on-the-fly stencil, (1,1,1) mask = no mask
    (numba_kernels._grad_at :188-212, _no_mask :314-317)."""
    f = _f32(f)
    stored = np.shape(gx) == f.shape
    gx, gy, gz = (_f32(a) for a in (gx, gy, gz))
    m = np.ascontiguousarray(mask, dtype=np.uint8)
    m = m if m.shape == f.shape else None
    return f, gx, gy, gz, int(stored), m


def _split(n, split_index, split_keep):
    if split_index is None or split_keep is None:
        return None, None, 0
    si = np.ascontiguousarray(split_index, dtype=np.int64)
    sk = np.ascontiguousarray(split_keep, dtype=np.uint8)
    return si, sk, int(sk.shape[1]) if sk.ndim == 2 else 0


# --------------------------------------------------------------------------- interpolation / gradients
def znssd(f, g, coords, P, half, mode):
    """FP64 ZNSSD cost (N,) of the residual numba_kernels.py:705-708 per subset under warps P (N,12)."""
    f, g = _f32(f), _f32(g)
    coords = np.ascontiguousarray(coords, dtype=np.int64)
    P = np.ascontiguousarray(P, dtype=np.float64).reshape(-1, 12)
    out = np.empty(coords.shape[0])
    hx, hy, hz = (int(h) for h in half)
    lib().orc_znssd(_ptr(f), _ptr(g), *f.shape, _ptr(coords), coords.shape[0], hx, hy, hz, int(mode), _ptr(P), _ptr(out))
    return out


BSPLINE_POLE = np.sqrt(3.0) - 2.0
BSPLINE_HALF_TAPS = 32


def bspline_weights() -> np.ndarray:
    """Taps sqrt(3) z^j, j = 0..32, of the cubic B-spline prefilter (the inverse of (z + 4 + 1/z) / 6)."""
    return np.sqrt(3.0) * BSPLINE_POLE ** np.arange(BSPLINE_HALF_TAPS + 1)


def gaussian_weights(sigma: float) -> np.ndarray:
    """Taps j = 0..r, r = int(4 sigma + 0.5), of the normalised Gaussian (scipy.ndimage.gaussian_filter, truncate 4)."""
    r = int(4.0 * float(sigma) + 0.5)
    x = np.arange(-r, r + 1)
    phi = np.exp(-0.5 / (float(sigma) * float(sigma)) * x**2)
    phi = phi / phi.sum()
    return np.ascontiguousarray(phi[r:])


def sep_filter(vol, axis, w, boundary):
    """One axis (0 = x, 1 = y, 2 = z) of a symmetric FIR, FP64 sums, float32 out; boundary 0 mirror, 1 nearest."""
    v = _f32(vol)
    w = np.ascontiguousarray(w, dtype=np.float64)
    out = np.empty_like(v)
    nz, ny, nx = v.shape
    lib().orc_sep_filter(_ptr(v), _ptr(out), nz, ny, nx, int(axis), _ptr(w), len(w) - 1, int(boundary))
    return out


def prefilter_bspline(vol):
    """io/volume_ops.py:215-222: cubic B-spline coefficients, mirror boundary.  Axes z, y, x in turn, each rounded
    to float32, the order in which scipy.ndimage filters array axes 0, 1, 2."""
    out = _f32(vol)
    for axis in (2, 1, 0):
        out = sep_filter(out, axis, bspline_weights(), 0)
    return out


def presmooth_volume(vol, sigma):
    """io/volume_ops.py:200-212: Gaussian smoothing with edge repeat (axes z, y, x in turn), identity when
    sigma <= 0."""
    if sigma is None or sigma <= 0:
        return _f32(vol)
    out = _f32(vol)
    for axis in (2, 1, 0):
        out = sep_filter(out, axis, gaussian_weights(sigma), 1)
    return out


def block_downsample(vol, factor):
    """integer_search.py:235-244: block means of factor^3 voxels (trailing voxels dropped), FP64 sums, float32."""
    v = np.asarray(vol, dtype=np.float32)
    if factor <= 1:
        return v.copy()
    nz, ny, nx = (s // factor * factor for s in v.shape)
    b = v[:nz, :ny, :nx].astype(np.float64).reshape(nz // factor, factor, ny // factor, factor, nx // factor, factor)
    return (b.sum(axis=(1, 3, 5)) / float(factor**3)).astype(np.float32)


def phase_correlation_shift(f, g, max_dim=128):
    """integer_search.py:247-291 without a VOI: block means until no axis exceeds max_dim, centring and a separable
    Hann window in float32, then the cross-power spectrum and its inverse in complex128; the first maximum,
    wrapped to (-n/2, n/2] and scaled back, as (dx, dy, dz)."""
    import math

    f = np.asarray(f, dtype=np.float32)
    g = np.asarray(g, dtype=np.float32)
    factor = max(1, int(math.ceil(max(f.shape) / max_dim)))
    fs, gs = block_downsample(f, factor), block_downsample(g, factor)
    fs = fs - np.float32(fs.astype(np.float64).mean())
    gs = gs - np.float32(gs.astype(np.float64).mean())
    win = np.ones(fs.shape, dtype=np.float32)
    for ax, n in enumerate(fs.shape):
        shape = [1, 1, 1]
        shape[ax] = n
        win = win * np.hanning(n).astype(np.float32).reshape(shape)
    Ff = np.fft.fftn((fs * win).astype(np.float64))
    Fg = np.fft.fftn((gs * win).astype(np.float64))
    R = Fg * np.conj(Ff)
    mag = np.abs(R)
    R = R / np.where(mag > 1e-12, mag, 1.0)
    r = np.real(np.fft.ifftn(R))
    shift = np.array(np.unravel_index(int(np.argmax(r)), r.shape), dtype=np.float64)
    for ax, n in enumerate(r.shape):
        if shift[ax] > n // 2:
            shift[ax] -= n
    dz, dy, dx = shift * factor
    return np.array([dx, dy, dz], dtype=np.float64)


def sample_points(vol, zs, ys, xs, mode):
    """interp_kernels.sample_points (:139-152)."""
    vol = _f32(vol)
    zs, ys, xs = (np.ascontiguousarray(a, dtype=np.float64) for a in (zs, ys, xs))
    out = np.empty(zs.shape[0])
    lib().orc_sample_points(_ptr(vol), *vol.shape, _ptr(zs), _ptr(ys), _ptr(xs), zs.shape[0], int(mode), _ptr(out))
    return out


def compute_gradients(f, border=3):
    """io/volume_ops._gradient_stencil7 (:124-155) / compute_gradients (:177-197)."""
    f = _f32(f)
    gx, gy, gz = (np.empty_like(f) for _ in range(3))
    lib().orc_gradients(_ptr(f), *f.shape, int(border), _ptr(gx), _ptr(gy), _ptr(gz))
    return gx, gy, gz


def compose_warp(P, dP):
    """numba_kernels.compose_warp_inplace (:145-180) on a copy."""
    P = np.array(P, dtype=np.float64)
    dP = np.ascontiguousarray(dP, dtype=np.float64)
    ok = lib().orc_compose_warp(_ptr(P), _ptr(dP))
    return P, bool(ok)


# --------------------------------------------------------------------------- local kernels
def precompute_nodes(coords, hx, hy, hz, f, gx, gy, gz, mask, min_valid_ratio, cond_max, stride=1, split_index=None,
                     split_keep=None):
    """numba_kernels.precompute_nodes (:499-509)."""
    coords = np.ascontiguousarray(coords, dtype=np.int64)
    N = coords.shape[0]
    f, gx, gy, gz, stored, m = _vol_args(f, gx, gy, gz, mask)
    si, sk, kb = _split(N, split_index, split_keep)
    H = np.zeros((N, 12, 12))
    L = np.zeros((N, 12, 12))
    mf = np.zeros(N)
    bf = np.ones(N)
    nv = np.zeros(N, dtype=np.int64)
    valid = np.zeros(N, dtype=np.uint8)
    lib().orc_precompute(_ptr(coords), N, int(hx), int(hy), int(hz), int(stride), _ptr(f), _ptr(gx), _ptr(gy), _ptr(gz), stored,
                         _ptr(m), *f.shape, _ptr(si), _ptr(sk), kb, float(min_valid_ratio), float(cond_max), _ptr(H), _ptr(L),
                         _ptr(mf), _ptr(bf), _ptr(nv), _ptr(valid))
    return H, L, mf, bf, nv, valid.astype(bool)


def icgn_12dof_parallel(coords, P0, hx, hy, hz, f, gx, gy, gz, mask, g, mode, L_all, meanf_all, bottomf_all, valid, tol, dp_tol,
                        max_iter, patience, stride=1, H_all=None, pattern=None, noise_gain=0.0, predictive=True,
                        split_index=None, split_keep=None):
    """numba_kernels.icgn_12dof_parallel (:1211-1278); meanf_all is unused there too (the statistics are dynamic)."""
    coords = np.ascontiguousarray(coords, dtype=np.int64)
    N = coords.shape[0]
    f, gx, gy, gz, stored, m = _vol_args(f, gx, gy, gz, mask)
    g = _f32(g)
    P0 = np.ascontiguousarray(P0, dtype=np.float64).reshape(N, 12)
    L_all = np.ascontiguousarray(L_all, dtype=np.float64)
    valid = np.ascontiguousarray(valid, dtype=np.uint8)
    use_noise = H_all is not None and pattern is not None and noise_gain > 0.0
    H_arr = np.ascontiguousarray(H_all, dtype=np.float64) if use_noise else None
    pat = np.ascontiguousarray(pattern, dtype=np.float64) if use_noise else None
    si, sk, kb = _split(N, split_index, split_keep)
    P_out = np.empty((N, 12))
    n_iter = np.zeros(N, dtype=np.int32)
    status = np.zeros(N, dtype=np.int8)
    zncc = np.zeros(N)
    lib().orc_icgn12(_ptr(coords), N, _ptr(P0), int(hx), int(hy), int(hz), int(stride), _ptr(f), _ptr(gx), _ptr(gy), _ptr(gz),
                     stored, _ptr(m), _ptr(g), *f.shape, int(mode), _ptr(L_all), _ptr(valid), float(tol), float(dp_tol),
                     int(max_iter), int(patience), _ptr(H_arr), _ptr(pat), float(noise_gain if use_noise else 0.0),
                     int(bool(predictive)), _ptr(si), _ptr(sk), kb, _ptr(P_out), _ptr(n_iter), _ptr(status), _ptr(zncc))
    return P_out, n_iter, status, zncc


def icgn_3dof_parallel(coords, U_old, F_fixed, vdual, hx, hy, hz, f, gx, gy, gz, mask, g, mode, H_all, meanf_all, bottomf_all,
                       valid, mu, tol, dp_tol, max_iter, patience, stride=1, n_full=0.0, noise_gain=0.0, predictive=True,
                       split_index=None, split_keep=None):
    """numba_kernels.icgn_3dof_parallel (:1281-1346)."""
    coords = np.ascontiguousarray(coords, dtype=np.int64)
    N = coords.shape[0]
    f, gx, gy, gz, stored, m = _vol_args(f, gx, gy, gz, mask)
    g = _f32(g)
    U_old = np.ascontiguousarray(U_old, dtype=np.float64).reshape(N, 3)
    F_fixed = np.ascontiguousarray(F_fixed, dtype=np.float64).reshape(N, 9)
    vdual = np.ascontiguousarray(vdual, dtype=np.float64).reshape(N, 3)
    H_all = np.ascontiguousarray(H_all, dtype=np.float64)
    bottomf_all = np.ascontiguousarray(bottomf_all, dtype=np.float64)
    valid = np.ascontiguousarray(valid, dtype=np.uint8)
    si, sk, kb = _split(N, split_index, split_keep)
    U_out = np.empty((N, 3))
    n_iter = np.zeros(N, dtype=np.int32)
    status = np.zeros(N, dtype=np.int8)
    zncc = np.zeros(N)
    lib().orc_icgn3(_ptr(coords), N, _ptr(U_old), _ptr(F_fixed), _ptr(vdual), int(hx), int(hy), int(hz), int(stride), _ptr(f),
                    _ptr(gx), _ptr(gy), _ptr(gz), stored, _ptr(m), _ptr(g), *f.shape, int(mode), _ptr(H_all), _ptr(bottomf_all),
                    _ptr(valid), float(mu), float(tol), float(dp_tol), int(max_iter), int(patience), float(n_full),
                    float(noise_gain if noise_gain > 0.0 else 0.0), int(bool(predictive)), _ptr(si), _ptr(sk), kb, _ptr(U_out),
                    _ptr(n_iter), _ptr(status), _ptr(zncc))
    return U_out, n_iter, status, zncc


# --------------------------------------------------------------------------- integer search
def zncc_direct(f, g, coords, hx, hy, hz, rx, ry, rz, wx0, wy0, wz0, t_ok, out):
    """integer_search._zncc_direct (:44-151): fills ``out`` (n, vz, vy, vx) in place."""
    f, g = _f32(f), _f32(g)
    coords = np.ascontiguousarray(coords, dtype=np.int64)
    wx0, wy0, wz0 = (np.ascontiguousarray(a, dtype=np.int64) for a in (wx0, wy0, wz0))
    t_ok = np.ascontiguousarray(t_ok, dtype=np.uint8)
    buf = out if (out.dtype == np.float64 and out.flags.c_contiguous) else np.empty(out.shape)
    lib().orc_zncc_direct(_ptr(f), _ptr(g), *f.shape, _ptr(coords), coords.shape[0], int(hx), int(hy), int(hz), int(rx), int(ry),
                          int(rz), _ptr(wx0), _ptr(wy0), _ptr(wz0), _ptr(t_ok), _ptr(buf))
    if buf is not out:
        out[...] = buf


def _quadratic_pinv():
    """Pseudo-inverse of the 27-point quadratic design (integer_search.py:210-227)."""
    dz, dy, dx = np.meshgrid([-1, 0, 1], [-1, 0, 1], [-1, 0, 1], indexing="ij")
    dx, dy, dz = dx.ravel().astype(float), dy.ravel().astype(float), dz.ravel().astype(float)
    D = np.column_stack([np.ones(27), dx, dy, dz, dx * dy, dx * dz, dy * dz, dx**2, dy**2, dz**2])
    return np.linalg.pinv(D)


_PINV = _quadratic_pinv()
_NB = [a.ravel()[None, :] for a in np.meshgrid([-1, 0, 1], [-1, 0, 1], [-1, 0, 1], indexing="ij")]


def subvoxel_peak(neigh):
    """integer_search._subvoxel_peak (:297-321)."""
    n = neigh.shape[0]
    coef = neigh @ _PINV.T
    a = coef[:, 1:4]
    H = np.empty((n, 3, 3))
    H[:, 0, 0] = 2 * coef[:, 7]
    H[:, 1, 1] = 2 * coef[:, 8]
    H[:, 2, 2] = 2 * coef[:, 9]
    H[:, 0, 1] = H[:, 1, 0] = coef[:, 4]
    H[:, 0, 2] = H[:, 2, 0] = coef[:, 5]
    H[:, 1, 2] = H[:, 2, 1] = coef[:, 6]
    out = np.zeros((n, 3))
    det = np.linalg.det(H)
    ok = np.abs(det) > 1e-12
    if ok.any():
        sol = np.linalg.solve(H[ok], -a[ok][:, :, None])[:, :, 0]
        good = np.all(np.abs(sol) <= 1.0, axis=1) & np.all(np.isfinite(sol), axis=1)
        tmp = np.zeros((int(ok.sum()), 3))
        tmp[good] = sol[good]
        out[ok] = tmp
    return out


# integer_search.py:41, :395: above this many offset x template-voxel products per node the reference's CPU
# search takes its FFT branch
DIRECT_NCC_MAX_OPS = 3.0e7


def window_box_stats(W, sz, sy, sx):
    """integer_search._window_box_stats (:154-207): sums of W and of its float32 squares over every template box
    of each node's window W (n, wz, wy, wx), FP64 summed-area tables; returns (sum, sq), (n, vz, vy, vx) each."""
    W = np.ascontiguousarray(W, dtype=np.float32)
    n, wz, wy, wx = W.shape
    shape = (n, wz - sz + 1, wy - sy + 1, wx - sx + 1)
    s1, s2 = np.empty(shape), np.empty(shape)
    lib().orc_window_box_stats(_ptr(W), n, wz, wy, wx, int(sz), int(sy), int(sx), _ptr(s1), _ptr(s2))
    return s1, s2


def ncc_maps_fft(f, g, coords, half, radius, wx0, wy0, wz0):
    """The FFT branch of integer_search.ncc_search (:418-443) for the nodes ``coords`` (templates inside f):
    float32 windows and mean-removed float32 templates, their real FFTs over the 2,3,5-smooth padded box
    (scipy.fft, as the reference), the product with the conjugate template spectrum, its inverse cropped to
    the valid offsets, normalised by the FP64 window box statistics and the template norm, clipped to [-1, 1].
    Returns (maps (n, vz, vy, vx) float64, template norms (n,))."""
    from scipy import fft as sfft

    hx, hy, hz = half
    rx, ry, rz = radius
    sx, sy, sz = 2 * hx + 1, 2 * hy + 1, 2 * hz + 1
    wx, wy, wz = sx + 2 * rx, sy + 2 * ry, sz + 2 * rz
    vx, vy, vz = 2 * rx + 1, 2 * ry + 1, 2 * rz + 1
    n = coords.shape[0]
    box = tuple(sfft.next_fast_len(int(w), real=True) for w in (wz, wy, wx))
    T = np.empty((n, sz, sy, sx), dtype=np.float32)
    W = np.empty((n, wz, wy, wx), dtype=np.float32)
    for k in range(n):
        x, y, z = (int(a) for a in coords[k])
        T[k] = f[z - hz:z + hz + 1, y - hy:y + hy + 1, x - hx:x + hx + 1]
        W[k] = g[wz0[k]:wz0[k] + wz, wy0[k]:wy0[k] + wy, wx0[k]:wx0[k] + wx]
    # template mean in FP64, subtracted in float32; its norm in FP64
    T -= T.mean(axis=(1, 2, 3), dtype=np.float64, keepdims=True).astype(np.float32)
    t_norm = np.sqrt((T.astype(np.float64) ** 2).sum(axis=(1, 2, 3)))
    spec = sfft.rfftn(W, s=box, axes=(1, 2, 3), workers=-1)
    spec *= np.conj(sfft.rfftn(T, s=box, axes=(1, 2, 3), workers=-1))
    cross = sfft.irfftn(spec, s=box, axes=(1, 2, 3), workers=-1)[:, :vz, :vy, :vx].astype(np.float64)
    s1, s2 = window_box_stats(W, sz, sy, sx)
    var = np.maximum(s2 - s1 * s1 / float(sx * sy * sz), 0.0)
    denom = np.sqrt(var) * t_norm[:, None, None, None]
    maps = np.zeros_like(cross)
    np.divide(cross, denom, out=maps, where=denom > 1e-10)
    np.clip(maps, -1.0, 1.0, out=maps)
    return maps, t_norm


def ncc_engine(half, radius) -> str:
    """The reference CPU search's engine for a template half-width and radius (integer_search.py:395)."""
    n_tpl = np.prod([2 * int(h) + 1 for h in half])
    n_off = np.prod([2 * int(r) + 1 for r in radius])
    return "direct" if n_tpl * n_off <= DIRECT_NCC_MAX_OPS else "fft"


def ncc_search(f, g, coords, subset, radius, shift0=None, engine="direct"):
    """integer_search.ncc_search (:329-483).  ``engine``: "direct" (the FP64 map of _zncc_direct for every
    size: the exact-arithmetic map), "fft" (the reference's FP32 FFT branch) or "auto" (the reference's own
    switch, ``ncc_engine``)."""
    f, g = _f32(f), _f32(g)
    nz, ny, nx = f.shape
    coords = np.asarray(coords, dtype=np.int64)
    N = coords.shape[0]
    hx, hy, hz = (int(w) // 2 for w in subset)
    rx, ry, rz = (int(r) for r in radius)
    sx, sy, sz = 2 * hx + 1, 2 * hy + 1, 2 * hz + 1
    wx, wy, wz = sx + 2 * rx, sy + 2 * ry, sz + 2 * rz
    if engine == "auto":
        engine = ncc_engine((hx, hy, hz), (rx, ry, rz))
    if engine not in ("direct", "fft"):
        raise ValueError(f"unknown NCC engine {engine!r}")
    if shift0 is None:
        shift0 = np.zeros((N, 3), dtype=np.int64)
    shift0 = np.asarray(np.round(shift0), dtype=np.int64)
    disp = np.full((N, 3), np.nan)
    cc = np.full(N, np.nan)
    pce = np.full(N, np.nan)
    clipped = np.zeros(N, dtype=bool)
    ok = np.zeros(N, dtype=bool)
    out = {"disp": disp, "cc": cc, "pce": pce, "clipped": clipped, "ok": ok, "engine": engine}
    if wx > nx or wy > ny or wz > nz:
        return out
    cx, cy, cz = coords[:, 0], coords[:, 1], coords[:, 2]
    t_ok = (cx - hx >= 0) & (cx + hx < nx) & (cy - hy >= 0) & (cy + hy < ny) & (cz - hz >= 0) & (cz + hz < nz)
    dx0 = cx + shift0[:, 0] - hx - rx
    dy0 = cy + shift0[:, 1] - hy - ry
    dz0 = cz + shift0[:, 2] - hz - rz
    wx0 = np.clip(dx0, 0, nx - wx)
    wy0 = np.clip(dy0, 0, ny - wy)
    wz0 = np.clip(dz0, 0, nz - wz)
    free_lo = np.column_stack([dx0 >= 0, dy0 >= 0, dz0 >= 0])
    free_hi = np.column_stack([dx0 <= nx - wx, dy0 <= ny - wy, dz0 <= nz - wz])
    idx_all = np.flatnonzero(t_ok)
    vz, vy, vx = 2 * rz + 1, 2 * ry + 1, 2 * rx + 1
    chunk = 4096 if engine == "direct" else 64
    for start in range(0, idx_all.size, chunk):
        ids = idx_all[start:start + chunk]
        n = ids.size
        if engine == "direct":
            ncc = np.empty((n, vz, vy, vx))
            zncc_direct(f, g, coords[ids], hx, hy, hz, rx, ry, rz, wx0[ids], wy0[ids], wz0[ids], np.ones(n, dtype=bool), ncc)
            t_norm = np.where(ncc[:, 0, 0, 0] > -1.5, 1.0, 0.0)  # a flat template marks its whole map -2
            ncc[ncc < -1.0] = 0.0
        else:
            ncc, t_norm = ncc_maps_fft(f, g, coords[ids], (hx, hy, hz), (rx, ry, rz), wx0[ids], wy0[ids], wz0[ids])
        flat = ncc.reshape(n, -1)
        pk = np.argmax(flat, axis=1)
        pz, py, px = np.unravel_index(pk, ncc.shape[1:])
        peak_val = flat[np.arange(n), pk]
        cmin = flat - flat.min(axis=1, keepdims=True)
        energy = np.mean(cmin * cmin, axis=1)
        pk_min = cmin[np.arange(n), pk]
        pce_k = np.divide(pk_min * pk_min, energy, out=np.zeros(n), where=energy > 1e-30)
        lo, hi = free_lo[ids], free_hi[ids]
        if rx > 0 or ry > 0 or rz > 0:
            on_edge = (((px == 0) & lo[:, 0]) | ((px == 2 * rx) & hi[:, 0]) | ((py == 0) & lo[:, 1]) | ((py == 2 * ry) & hi[:, 1])
                       | ((pz == 0) & lo[:, 2]) | ((pz == 2 * rz) & hi[:, 2]))
        else:
            on_edge = np.zeros(n, dtype=bool)
        sub = np.zeros((n, 3))
        at_border = (px == 0) | (px == 2 * rx) | (py == 0) | (py == 2 * ry) | (pz == 0) | (pz == 2 * rz)
        interior = ~at_border & (rx > 0) & (ry > 0) & (rz > 0)
        if interior.any():
            ii = np.flatnonzero(interior)
            neigh = ncc[ii[:, None], pz[ii][:, None] + _NB[0], py[ii][:, None] + _NB[1], px[ii][:, None] + _NB[2]]
            sub[ii] = subvoxel_peak(neigh)
        disp[ids, 0] = wx0[ids] + px + hx - cx[ids] + sub[:, 0]
        disp[ids, 1] = wy0[ids] + py + hy - cy[ids] + sub[:, 1]
        disp[ids, 2] = wz0[ids] + pz + hz - cz[ids] + sub[:, 2]
        cc[ids] = peak_val
        pce[ids] = pce_k
        clipped[ids] = on_edge
        ok[ids] = np.isfinite(peak_val) & (t_norm > 1e-10)
    disp[~ok] = np.nan
    return out


def ncc_search_expanding(f, g, coords, subset, radius, shift0=None, auto_expand=True, max_expand=3, engine="direct"):
    """integer_search.ncc_search_expanding (:486-524); ``engine`` as in ``ncc_search`` (each radius picks its own
    engine under "auto", as the reference's searches do)."""
    res = ncc_search(f, g, coords, subset, radius, shift0, engine)
    res["expansions"] = 0
    res["radius"] = tuple(int(r) for r in radius)
    rad = res["radius"]
    for _ in range(max_expand if auto_expand else 0):
        sel = res["clipped"] & res["ok"]
        n_ok = int(res["ok"].sum())
        if n_ok == 0 or sel.sum() <= 0.05 * n_ok:
            break
        rad = tuple(2 * r for r in rad)
        sub_shift = None if shift0 is None else np.asarray(shift0)[sel]
        sub = ncc_search(f, g, coords[sel], subset, rad, sub_shift, engine)
        if not sub["ok"].any():
            break
        idx = np.flatnonzero(sel)[sub["ok"]]
        for key in ("disp", "cc", "pce", "clipped", "ok"):
            res[key][idx] = sub[key][sub["ok"]]
        res["expansions"] += 1
        res["radius"] = rad
    return res


# --------------------------------------------------------------------------- global step (hex8 FEM)
_HEX8_SIGNS = np.array([[-1, -1, -1], [1, -1, -1], [1, 1, -1], [-1, 1, -1], [-1, -1, 1], [1, -1, 1], [1, 1, 1], [-1, 1, 1]],
                       dtype=np.float64)


def hex8_box_matrices(spacing, order=2):
    """mesh/hex8.hex8_box_matrices (:74-105): element K, M, G_j of an axis-aligned box."""
    if order == 1:
        p1, w1 = np.array([0.0]), np.array([2.0])
    elif order == 2:
        gp = 1.0 / np.sqrt(3.0)
        p1, w1 = np.array([-gp, gp]), np.array([1.0, 1.0])
    elif order == 3:
        gp = np.sqrt(3.0 / 5.0)
        p1, w1 = np.array([-gp, 0.0, gp]), np.array([5.0 / 9.0, 8.0 / 9.0, 5.0 / 9.0])
    else:
        raise ValueError(order)
    hx, hy, hz = (float(s) for s in spacing)
    inv_jac = np.diag([2.0 / hx, 2.0 / hy, 2.0 / hz])
    det_j = (hx / 2.0) * (hy / 2.0) * (hz / 2.0)
    s = _HEX8_SIGNS
    K = np.zeros((8, 8))
    M = np.zeros((8, 8))
    G = np.zeros((3, 8, 8))
    for k, wk in zip(p1, w1):
        for j, wj in zip(p1, w1):
            for i, wi in zip(p1, w1):
                ksi, eta, zeta = i, j, k
                N = 0.125 * (1 + s[:, 0] * ksi) * (1 + s[:, 1] * eta) * (1 + s[:, 2] * zeta)
                dN = np.empty((8, 3))
                dN[:, 0] = 0.125 * s[:, 0] * (1 + s[:, 1] * eta) * (1 + s[:, 2] * zeta)
                dN[:, 1] = 0.125 * (1 + s[:, 0] * ksi) * s[:, 1] * (1 + s[:, 2] * zeta)
                dN[:, 2] = 0.125 * (1 + s[:, 0] * ksi) * (1 + s[:, 1] * eta) * s[:, 2]
                dN = dN @ inv_jac
                wj_ = wi * wj * wk * det_j
                K += wj_ * (dN @ dN.T)
                M += wj_ * np.outer(N, N)
                for a in range(3):
                    G[a] += wj_ * np.outer(dN[:, a], N)
    return {"K": K, "M": M, "G": G}


def grid_elements(grid_shape):
    """mesh/grid_mesh.mesh_setup element connectivity (:79-103), node n = iz*ny*nx + iy*nx + ix."""
    nz, ny, nx = grid_shape
    iz, iy, ix = (a.ravel() for a in np.meshgrid(np.arange(nz - 1), np.arange(ny - 1), np.arange(nx - 1), indexing="ij"))

    def nid(a, b, c):
        return c * ny * nx + b * nx + a

    return np.column_stack([nid(ix, iy, iz), nid(ix + 1, iy, iz), nid(ix + 1, iy + 1, iz), nid(ix, iy + 1, iz),
                            nid(ix, iy, iz + 1), nid(ix + 1, iy, iz + 1), nid(ix + 1, iy + 1, iz + 1),
                            nid(ix, iy + 1, iz + 1)]).astype(np.int64)


def fem_operators(grid_shape, spacing, elem_active=None, order=2):
    """global_operators.build_fem_operators (:58-71) over the active elements."""
    n = int(np.prod(grid_shape))
    elems = grid_elements(grid_shape)
    if elem_active is not None:
        elems = elems[np.asarray(elem_active, dtype=bool)]
    box = hex8_box_matrices(spacing, order)

    def scatter(Ke):
        E = elems.shape[0]
        rows = np.broadcast_to(elems[:, :, None], (E, 8, 8)).ravel()
        cols = np.broadcast_to(elems[:, None, :], (E, 8, 8)).ravel()
        vals = np.broadcast_to(Ke[None], (E, 8, 8)).ravel()
        return sparse.coo_matrix((vals, (rows, cols)), shape=(n, n)).tocsr()

    Kg, M = scatter(box["K"]), scatter(box["M"])
    G = tuple(scatter(box["G"][j]) for j in range(3))
    mL = np.asarray(M.sum(axis=1)).ravel()
    active = np.zeros(n, dtype=bool)
    active[np.unique(elems)] = True
    return {"Kg": Kg, "M": M, "G": G, "mL": mL, "active": active, "n_nodes": n}


def global_system(ops, beta, mu, alpha=0.0):
    """subpb2_solver.build_global_system (:45-74), PCG branch."""
    A_full = ((beta + alpha) * ops["Kg"] + mu * ops["M"]).tocsr()
    act = np.flatnonzero(ops["active"])
    A = A_full[act][:, act].tocsr()
    d = A.diagonal()
    inv_diag = np.where(np.abs(d) > 1e-300, 1.0 / d, 1.0)
    return {"A": A, "inv_diag": inv_diag, "active_idx": act, "beta": beta, "mu": mu, "alpha": alpha, "ops": ops}


def pcg_multi(A, B, inv_diag, tol, max_iter, X0=None):
    """subpb2_solver.pcg_multi (:77-108): Jacobi-PCG for several right-hand sides."""
    X = np.zeros_like(B) if X0 is None else X0.copy()
    R = B - A @ X
    Z = inv_diag[:, None] * R
    P = Z.copy()
    rz = np.einsum("ij,ij->j", R, Z)
    bnorm = np.linalg.norm(B, axis=0)
    bnorm[bnorm == 0] = 1.0
    it = 0
    for it in range(1, max_iter + 1):
        AP = A @ P
        denom = np.einsum("ij,ij->j", P, AP)
        denom[denom == 0] = np.inf
        alpha = rz / denom
        X += P * alpha
        R -= AP * alpha
        if np.all(np.linalg.norm(R, axis=0) / bnorm < tol):
            break
        Z = inv_diag[:, None] * R
        rz_new = np.einsum("ij,ij->j", R, Z)
        beta = rz_new / np.where(rz == 0, np.inf, rz)
        P = Z + P * beta
        rz = rz_new
    return X, it


def global_rhs(ops, beta, mu, alpha, U1, F1, W, v):
    """subpb2_solver.global_rhs (:111-130)."""
    n = ops["n_nodes"]
    FmW = np.asarray(F1, dtype=np.float64).reshape(n, 3, 3) - np.asarray(W, dtype=np.float64).reshape(n, 3, 3)
    Umv = np.asarray(U1, dtype=np.float64).reshape(n, 3) - np.asarray(v, dtype=np.float64).reshape(n, 3)
    b = mu * (ops["M"] @ Umv)
    for j in range(3):
        b += beta * (ops["G"][j] @ FmW[:, :, j])
    if alpha != 0.0:
        b += alpha * (ops["Kg"] @ np.asarray(U1, dtype=np.float64).reshape(n, 3))
    return b


def solve_subpb2(system, U1, F1, W, v, tol=1e-8, max_iter=500):
    """subpb2_solver.solve_subpb2 (:133-155) with the PCG solver."""
    ops = system["ops"]
    b = global_rhs(ops, system["beta"], system["mu"], system["alpha"], U1, F1, W, v)
    U1 = np.asarray(U1, dtype=np.float64).reshape(ops["n_nodes"], 3)
    act = system["active_idx"]
    X, it = pcg_multi(system["A"], b[act], system["inv_diag"], tol, max_iter, X0=U1[act])
    U2 = U1.copy()
    U2[act] = X
    return U2, it


def nodal_gradient(ops, U):
    """global_operators.nodal_gradient (:151-170), FEM branch: F_ij = (G_j^T u_i) / m_L, NaN off the active set."""
    n = ops["n_nodes"]
    U = np.asarray(U, dtype=np.float64).reshape(n, 3)
    F = np.empty((n, 3, 3))
    safe = np.where(ops["mL"] > 1e-15, ops["mL"], 1.0)
    for j in range(3):
        GT = ops["G"][j].T
        for i in range(3):
            F[:, i, j] = (GT @ U[:, i]) / safe
    F[~ops["active"]] = np.nan
    return F


# --------------------------------------------------------------------------- volume normalisation
def normalize_volume(vol):
    """io/volume_ops.normalize_volume (:105-121) over the whole volume, on the path the reference takes for
    integer and float inputs of two or more bytes: moments of (v - pilot) per z slice in FP64, accumulated in
    C order with the voxel kept in its own precision before the subtraction (voi_mean_std :79-99,
    _voi_moments :52-68), the slice totals summed, then float32((v - mean) / std) (_normalize_into :71-76)."""
    a = np.ascontiguousarray(vol)
    nz, ny, nx = a.shape
    pilot = float(a[nz // 2, ny // 2, nx // 2])
    d = a.reshape(nz, -1).astype(np.float64) - pilot
    s = np.add.accumulate(d, axis=1)[:, -1]  # sequential per slice, like the reference's inner loops
    ss = np.add.accumulate(d * d, axis=1)[:, -1]
    n = float(a.size)
    mean_shift = s.sum() / n
    var = max(ss.sum() / n - mean_shift * mean_shift, 0.0)
    mean, std = pilot + mean_shift, float(np.sqrt(var))
    if std < 1e-12:
        std = 1.0
    return ((a.astype(np.float64) - mean) * (1.0 / std)).astype(np.float32)


# --------------------------------------------------------------------------- node-grid post-processing
def _neighbour_footprint():
    fp = np.ones((3, 3, 3), dtype=bool)
    fp[1, 1, 1] = False  # the 26 neighbours, the node itself left out
    return fp


def fill_nan_grid(grid):
    """utils/inpaint.fill_nan_grid (:35-128), spring model on a (nz, ny, nx) grid: the unknown (NaN) nodes solve
    the discrete Laplace equation with their six grid neighbours, known neighbours entering as Dirichlet data,
    plus a 1e-10 Tikhonov term; a sparse direct solve (conjugate gradients above 60,000 unknowns).  All NaN:
    zeros."""
    from scipy.sparse.linalg import cg, spsolve

    arr = np.array(grid, dtype=np.float64, copy=True)
    unk = np.isnan(arr)
    m = int(unk.sum())
    if m == 0:
        return arr
    if unk.all():
        return np.zeros_like(arr)
    flat = arr.ravel()
    pos = np.full(flat.size, -1, dtype=np.int64)
    pos[np.flatnonzero(unk.ravel())] = np.arange(m)
    ids = np.arange(flat.size).reshape(arr.shape)
    deg = np.zeros(m)
    rhs = np.zeros(m)
    rows, cols = [], []
    for ax in range(arr.ndim):
        if arr.shape[ax] < 2:
            continue
        lo = ids.take(np.arange(arr.shape[ax] - 1), axis=ax).ravel()
        hi = ids.take(np.arange(1, arr.shape[ax]), axis=ax).ravel()
        for p, q in ((lo, hi), (hi, lo)):  # each grid edge couples both of its ends
            pu = pos[p]
            e = pu >= 0
            pu, qn = pu[e], q[e]
            np.add.at(deg, pu, 1.0)
            qu = pos[qn]
            kn = qu < 0
            np.add.at(rhs, pu[kn], flat[qn[kn]])
            rows.append(pu[~kn])
            cols.append(qu[~kn])
    r = np.concatenate(rows + [np.arange(m)])
    c = np.concatenate(cols + [np.arange(m)])
    v = np.concatenate([-np.ones(r.size - m), deg])
    A = sparse.coo_matrix((v, (r, c)), shape=(m, m)).tocsr() + sparse.eye(m, format="csr") * 1e-10
    if m <= 60_000:
        x = spsolve(A.tocsc(), rhs)
    else:
        x, info = cg(A, rhs, rtol=1e-10, maxiter=2000)
        if info != 0:
            x = spsolve(A.tocsc(), rhs)
    flat[np.flatnonzero(unk.ravel())] = x
    return flat.reshape(arr.shape)


def median_test(field, valid, threshold, eps=0.1):
    """utils/outlier_detection.universal_median_test (:135-163) on an uncut grid: per component, invalid nodes
    inpainted (fill_nan_grid), the normalised fluctuation |u - med26(u)| / (med26(|u - med26(u)|) + eps) over the
    26-neighbourhood (scipy median filter, nearest edges), 0 at invalid nodes; a valid node is an outlier when
    the norm of its component fluctuations exceeds ``threshold``.  field (nz, ny, nx, C) -> (nz, ny, nx) bool."""
    from scipy.ndimage import median_filter

    arr = np.asarray(field, dtype=np.float64)
    if arr.ndim == 3:
        arr = arr[..., None]
    if threshold <= 0:
        return np.zeros(arr.shape[:3], dtype=bool)
    fp = _neighbour_footprint()
    mag2 = np.zeros(arr.shape[:3])
    for k in range(arr.shape[3]):
        a = arr[..., k].copy()
        if valid is not None:
            a[~valid] = np.nan
        holes = np.isnan(a)
        if holes.all():
            continue
        if holes.any():
            a = fill_nan_grid(a)
        fl = a - median_filter(a, footprint=fp, mode="nearest")
        nf = np.abs(fl) / (median_filter(np.abs(fl), footprint=fp, mode="nearest") + eps)
        nf[holes] = 0.0
        mag2 += nf * nf
    flag = np.sqrt(mag2) > threshold
    if valid is not None:
        flag &= valid
    return flag


def _fill_bad(values, bad, grid_shape):
    """Every column of ``values`` (N, C) with the ``bad`` rows inpainted on the node grid (local_icgn.fill_bad_nodes
    :492-522, init_disp.clean_initial_guess :183-188); all bad: zeros."""
    if not bad.any():
        return values.copy()
    if bad.all():
        return np.zeros_like(values)
    out = values.copy()
    for k in range(values.shape[1]):
        comp = values[:, k].reshape(grid_shape).copy()
        comp[bad.reshape(grid_shape)] = np.nan
        out[:, k] = fill_nan_grid(comp).ravel()
    return out


def _outliers(values, bad, grid_shape, threshold):
    """The median test of the good nodes after a local pass, run only with more than 27 of them
    (local_icgn.py:466-475, subpb1_solver.py:140-149, init_disp.py:166-170)."""
    good = ~bad
    if threshold <= 0 or good.sum() <= 27:
        return np.zeros_like(bad)
    return median_test(values.reshape(tuple(grid_shape) + (values.shape[1],)), good.reshape(grid_shape), threshold).ravel()


def subset_valid_fraction(mask, coords, half):
    """mesh/grid_mesh.subset_valid_fraction (:139-186): mask voxels inside each node's box clipped to the volume,
    over the nominal box volume."""
    m = np.asarray(mask) != 0
    nz, ny, nx = m.shape
    sat = np.zeros((nz + 1, ny + 1, nx + 1), dtype=np.int64)
    sat[1:, 1:, 1:] = m.cumsum(0).cumsum(1).cumsum(2)
    hx, hy, hz = half
    cx, cy, cz = (np.asarray(coords[:, k], dtype=np.int64) for k in range(3))
    x0, x1 = np.clip(cx - hx, 0, nx), np.clip(cx + hx + 1, 0, nx)
    y0, y1 = np.clip(cy - hy, 0, ny), np.clip(cy + hy + 1, 0, ny)
    z0, z1 = np.clip(cz - hz, 0, nz), np.clip(cz + hz + 1, 0, nz)
    cnt = (sat[z1, y1, x1] - sat[z0, y1, x1] - sat[z1, y0, x1] - sat[z1, y1, x0] + sat[z0, y0, x1] + sat[z0, y1, x0]
           + sat[z1, y0, x0] - sat[z0, y0, x0])
    return cnt / float((2 * hx + 1) * (2 * hy + 1) * (2 * hz + 1))


# --------------------------------------------------------------------------- one full AL-DVC pass
PASS_DEFAULTS = dict(winsize=(32, 32, 32), search_radius=(8, 8, 8), init_subset=None, interp_method="cubic", subset_stride=1,
                     icgn_tol=1e-2, icgn_dp_tol=1e-3, icgn_max_iter=100, icgn_patience=5, icgn_predictive_stop=True,
                     min_valid_ratio=0.5, hessian_cond_max=1e12, init_outlier_threshold=2.0, local_outlier_threshold=2.0,
                     ncc_auto_expand=True, ncc_max_expand=3, init_min_pce=0.0, use_global_step=True, mu=1e-3, beta=1e-3,
                     alpha=0.0, admm_max_iter=4, admm_tol=1e-2, dual_update="accumulate", pcg_tol=1e-8, pcg_max_iter=500,
                     gauss_pt_order=2, ncc_engine="auto")


def aldvc_pass(f, g, coords, grid_shape, spacing, mask=None, node_half=None, **prm):
    """One frame pair of core/pipeline.run_aldvc (:255-366) in FP64 on normalised volumes f, g: sections 3-6 with
    the "ncc" initial guess and no global pre-shift, a fixed beta, the FEM global step and the PCG solver.

    - reference-frame validity (grid_mesh.apply_mask_to_mesh :191-253 with a boolean ``mask``; precompute
      validity, local_icgn.precompute_local_context :223-347, which then becomes the mesh's node validity);
    - initial guess (init_disp.compute_initial_guess :53-140, clean_initial_guess :143-189): NCC search with
      radius expansion over the valid nodes, failed / invalid / outlying nodes inpainted;
    - local 12-DOF IC-GN (local_icgn.local_icgn :398-489): non-converged and outlying nodes inpainted, U and F;
    - global step (subpb2_solver.solve_subpb2 :133-155, global_operators.nodal_gradient :151-170), non-finite F
      replaced by the local F (pipeline.py:300-310);
    - ADMM steps 2..admm_max_iter (pipeline.py:316-352): 3-DOF subproblem 1 (subpb1_solver.subpb1_solver
      :77-164: rejected nodes keep the global estimate), global step, dual update, early stop on the RMS
      updates.

    ``node_half`` (N, 3) gives per-node subset half-widths (uneven subsets, every one within ``winsize``): each
    shape's nodes run through the kernels together, as the reference runs one shape per call, and validity
    uses each node's own box.  Returns a dict of per-node arrays and scalars."""
    p = dict(PASS_DEFAULTS)
    unknown = set(prm) - set(p)
    if unknown:
        raise TypeError(f"unknown pass parameters {sorted(unknown)}")
    p.update(prm)
    f, g = _f32(f), _f32(g)
    grid_shape = tuple(int(s) for s in grid_shape)
    coords = np.asarray(coords, dtype=np.int64)
    N = coords.shape[0]
    half = tuple(int(w) // 2 for w in p["winsize"])
    halves = np.tile(np.asarray(half, dtype=np.int64), (N, 1)) if node_half is None else np.asarray(node_half, dtype=np.int64)
    mode = {"linear": 0, "cubic": 1, "bspline": 2}[p["interp_method"]]
    g_prep = prefilter_bspline(g) if mode == 2 else g
    gx, gy, gz = compute_gradients(f)
    m_u8 = np.ones((1, 1, 1), np.uint8) if mask is None else np.ascontiguousarray(mask, dtype=np.uint8)
    stride = int(p["subset_stride"])
    groups = [np.flatnonzero((halves == s).all(axis=1)) for s in np.unique(halves, axis=0)]

    # reference-frame node validity and the active elements
    if mask is None:
        node_valid = np.ones(N, dtype=bool)
    else:
        frac = np.empty(N)
        for sel in groups:
            frac[sel] = subset_valid_fraction(mask, coords[sel], tuple(halves[sel[0]]))
        node_valid = (np.asarray(mask)[coords[:, 2], coords[:, 1], coords[:, 0]] != 0) & (frac >= p["min_valid_ratio"])
    elem_active = node_valid[grid_elements(grid_shape)].all(axis=1)

    # precompute, per subset shape
    H = np.zeros((N, 12, 12))
    L = np.zeros((N, 12, 12))
    meanf = np.zeros(N)
    bottomf = np.ones(N)
    valid = np.zeros(N, dtype=bool)
    for sel in groups:
        hs = tuple(int(v) for v in halves[sel[0]])
        H[sel], L[sel], meanf[sel], bottomf[sel], _, v = precompute_nodes(coords[sel], *hs, f, gx, gy, gz, m_u8, p["min_valid_ratio"],
                                                                           p["hessian_cond_max"], stride)
        valid[sel] = v
    valid &= node_valid

    # section 3: initial guess over the valid nodes
    sub0 = p["init_subset"] if p["init_subset"] is not None else tuple(min(int(w), 16) for w in p["winsize"])
    act = np.flatnonzero(valid) if valid.any() else np.arange(N)
    res = ncc_search_expanding(f, g, coords[act], sub0, p["search_radius"], None, p["ncc_auto_expand"], p["ncc_max_expand"],
                               p["ncc_engine"])
    disp = np.full((N, 3), np.nan)
    ok = np.zeros(N, dtype=bool)
    pce = np.full(N, np.nan)
    disp[act], ok[act], pce[act] = res["disp"], res["ok"], res["pce"]
    bad0 = ~ok | ~np.isfinite(disp).all(axis=1) | ~valid
    if p["init_min_pce"] > 0:
        bad0 |= np.isfinite(pce) & (pce < p["init_min_pce"])
    d = np.where(bad0[:, None], np.nan, disp)
    bad0 |= _outliers(d, bad0, grid_shape, p["init_outlier_threshold"])
    U0 = _fill_bad(np.where(bad0[:, None], np.nan, disp), bad0, grid_shape)

    # section 4: local 12-DOF IC-GN
    P0 = np.zeros((N, 12))
    P0[:, 9:] = U0
    P = np.zeros((N, 12))
    it12 = np.zeros(N, dtype=np.int32)
    st12 = np.zeros(N, dtype=np.int8)
    zc12 = np.zeros(N)
    for sel in groups:
        hs = tuple(int(v) for v in halves[sel[0]])
        P[sel], it12[sel], st12[sel], zc12[sel] = icgn_12dof_parallel(
            coords[sel], P0[sel], *hs, f, gx, gy, gz, m_u8, g_prep, mode, L[sel], meanf[sel], bottomf[sel], valid[sel], p["icgn_tol"],
            p["icgn_dp_tol"], p["icgn_max_iter"], p["icgn_patience"], stride, predictive=p["icgn_predictive_stop"])
    bad = st12 != STATUS_CONVERGED
    bad |= _outliers(P[:, 9:], bad, grid_shape, p["local_outlier_threshold"])
    UF = _fill_bad(P, bad, grid_shape)
    U1, F1 = UF[:, 9:].copy(), UF[:, :9].reshape(N, 3, 3).copy()
    out = {"U0": U0, "init_bad": bad0, "ncc_radius": np.array(res["radius"]), "ncc_expansions": res["expansions"], "valid": valid,
           "node_valid": node_valid, "P_local": P, "status_local": st12, "n_iter_local": it12, "zncc_local": zc12,
           "U_local": U1.copy(), "F_local": F1.copy(), "U": U1, "F": F1, "status": st12, "zncc": zc12, "n_iter": it12,
           "admm_steps": 1}
    if not p["use_global_step"]:
        return out

    # sections 5-6: global step and ADMM
    ops = fem_operators(grid_shape, spacing, elem_active, p["gauss_pt_order"])
    system = global_system(ops, p["beta"], p["mu"], p["alpha"])

    def global_step(U1_, F1_, W_, v_):
        U2_, _ = solve_subpb2(system, U1_, F1_, W_, v_, p["pcg_tol"], p["pcg_max_iter"])
        F2_ = nodal_gradient(ops, U2_)
        return U2_, np.where(np.isfinite(F2_), F2_, F1_)

    W = np.zeros((N, 3, 3))
    v = np.zeros((N, 3))
    U2, F2 = global_step(U1, F1, W, v)
    W, v = F2 - F1, U2 - U1
    n_full = float(np.prod([(2 * h) // stride + 1 for h in half]))
    steps, st, zc, it = 1, st12, zc12, it12
    for step in range(2, int(p["admm_max_iter"]) + 1):
        steps = step
        U1_prev = U1
        U = np.zeros((N, 3))
        it = np.zeros(N, dtype=np.int32)
        st = np.zeros(N, dtype=np.int8)
        zc = np.zeros(N)
        for sel in groups:
            hs = tuple(int(x) for x in halves[sel[0]])
            U[sel], it[sel], st[sel], zc[sel] = icgn_3dof_parallel(
                coords[sel], U2[sel], F2[sel], v[sel], *hs, f, gx, gy, gz, m_u8, g_prep, mode, H[sel], meanf[sel], bottomf[sel],
                valid[sel], p["mu"], p["icgn_tol"], p["icgn_dp_tol"], p["icgn_max_iter"], p["icgn_patience"], stride, n_full=n_full,
                predictive=p["icgn_predictive_stop"])
        bad3 = st != STATUS_CONVERGED
        bad3 |= _outliers(U, bad3, grid_shape, p["local_outlier_threshold"])
        U1 = np.where(bad3[:, None], U2, U)
        F1 = F2
        U2n, F2n = global_step(U1, F1, W, v)
        du_g = float(np.sqrt(np.mean((U2n - U2) ** 2)))
        du_l = float(np.sqrt(np.mean((U1 - U1_prev) ** 2)))
        if p["dual_update"] == "accumulate":
            W, v = W + (F2n - F1), v + (U2n - U1)
        else:
            W, v = F2n - F1, U2n - U1
        U2, F2 = U2n, F2n
        if du_g < p["admm_tol"] or du_l < p["admm_tol"]:
            break
    out.update(U=U2, F=F2, status=st, zncc=zc, n_iter=it, admm_steps=steps)
    return out
