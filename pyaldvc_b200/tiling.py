"""The AL-DVC pass over boxes of the volume, the frames streamed from host memory one box at a time.

pyALDVC solver/tiling.py (TileBox :48-111, tile_pad :141-175, plan_tiles :204-289) and the per-box loops of
local_icgn.py:430-459 (12-DOF, with the escape retry), precompute_local_context :239-330 and
subpb1_solver.py:34-58 (3-DOF).  The local kernels address every volume relative to a node centre and never
reduce across nodes, so a block of nodes is solved against a box of the volumes with the box's origin subtracted
from its node coordinates.  The reference tiles its local steps only and keeps the normalised frames whole in
host memory; here every step that reads voxels runs box by box, so the device holds one box (about 41 bytes per
box voxel) and the frames stay in host memory, or a memory map, of any size:

- normalisation: the whole volume's FP64 moments accumulated slab by slab (``aldvc_volume_moments``), each box
  normalised with them (``aldvc_normalize_sums``); one slab gives exactly ``aldvc_normalize``'s statistics;
- Gaussian presmoothing and the B-spline prefilter: finite FIR filters (``aldvc_sep_filter``) run on the box grown
  by their reach, so the box's values are the whole-volume filter's (mirror and nearest boundaries see the same
  volume faces, and an open face's wrong values stay in the growth that is cut away);
- gradients: the 7-point stencil on the box; every reference window lies 3 voxels inside an open face;
- the global shift and the coarse pyramid levels: block means built slab by slab (whole blocks per slab);
- integer search: boxes holding each node's template and its volume-clamped search window, so the clamp in the
  box is the volume's; the radius expansion is decided over all nodes, as the reference does;
- precompute, 12-DOF and 3-DOF IC-GN: the reference's plan (halo from the displacement present), nodes that leave
  an open face of their box retried in boxes with a wider halo;
- median tests, inpainting, the global hex8 step and the ADMM updates: node arrays, whole on the device.

The 12-DOF and 3-DOF results differ from the untiled pass only by the rounding of ``x0 + P[9]`` with a
box-local ``x0`` (the reference's own tiling has the same property, tests/test_tiling.py:136-137).
"""

from __future__ import annotations

import math
import os
from concurrent.futures import ThreadPoolExecutor
from dataclasses import dataclass, field

import numpy as np
import torch

from . import autotune
from . import beta_tuning as BT
from . import integer_search as IS
from . import kernels as K
from . import pipeline as PL
from .mesh import surface_nodes

# tiling.py:33-38: the gradient stencil's reach beyond a reference window, and the highest sample offset a cubic
# interpolation touches beyond a deformed sample
REF_STENCIL_PAD = 3
SAMPLE_PAD = 2
MIN_TILE_NODES = 1
BSPLINE_REACH = K.BSPLINE_HALF_TAPS  # taps of the B-spline prefilter on each side
ESCAPE_RETRIES = 3  # wider halos tried for nodes that left an open face of their box
PAD_QUANTUM = 8  # halos of the pass rounded up to this, so that successive ADMM steps plan the same boxes
SLAB_VOXELS = 1 << 28  # voxels per slab of the whole-volume sweeps (normalisation moments, block means)
STATUS_OUT_OF_BOUNDS = 2


# --------------------------------------------------------------------------- geometry (tiling.py:48-111)
@dataclass(frozen=True)
class Box:
    """A sub-box of the volume: ``origin`` (z0, y0, x0) and ``shape`` (nz, ny, nx).  ``open_faces`` (-z +z -y +y -x
    +x) marks the faces cut by the tile rather than by the volume: a subset leaving through one of them means the
    halo was short, not that the node is out of bounds."""

    origin: tuple
    shape: tuple
    open_faces: tuple = (False,) * 6

    @property
    def slices(self) -> tuple:
        return tuple(slice(o, o + n) for o, n in zip(self.origin, self.shape))

    @property
    def is_whole(self) -> bool:
        return tuple(self.origin) == (0, 0, 0) and not any(self.open_faces)

    @property
    def has_open_face(self) -> bool:
        return any(self.open_faces)

    @property
    def n_voxels(self) -> int:
        return int(np.prod(self.shape))

    def crop(self, vol):
        """The box's voxels of a host array, contiguous (the array itself for a whole-volume box)."""
        if vol is None:
            return None
        if tuple(vol.shape) == tuple(self.shape):
            return vol
        return np.ascontiguousarray(vol[self.slices])

    def view(self, vol):
        """The box's voxels of a host array as a view (strided unless the box is the whole volume)."""
        return vol if tuple(vol.shape) == tuple(self.shape) else vol[self.slices]

    def shift(self, coords_xyz) -> np.ndarray:
        """``coords_xyz`` (N, 3) [x, y, z] in the box's frame."""
        z0, y0, x0 = self.origin
        return np.asarray(coords_xyz, dtype=np.int64) - np.array([x0, y0, z0], dtype=np.int64)[None, :]

    def contains_windows(self, coords_xyz, pad) -> bool:
        """Every node's window plus ``pad`` (px, py, pz) inside the box."""
        c = np.asarray(coords_xyz, dtype=np.int64)
        if c.size == 0:
            return True
        for axis, lo, n, p in ((0, self.origin[2], self.shape[2], pad[0]), (1, self.origin[1], self.shape[1], pad[1]),
                               (2, self.origin[0], self.shape[0], pad[2])):
            if int(c[:, axis].min()) - p < lo or int(c[:, axis].max()) + p > lo + n - 1:
                return False
        return True

    def grown(self, reach, volume_shape) -> tuple:
        """(the box grown by ``reach`` (rz, ry, rx) voxels on every side, clamped to the volume; the box's slices
        inside it)."""
        lo = [max(0, o - r) for o, r in zip(self.origin, reach)]
        hi = [min(int(s), o + n + r) for o, n, r, s in zip(self.origin, self.shape, reach, volume_shape)]
        big = Box(tuple(lo), tuple(h - l_ for h, l_ in zip(hi, lo)))
        inner = tuple(slice(o - l_, o - l_ + n) for o, l_, n in zip(self.origin, lo, self.shape))
        return big, inner


def whole_box(shape) -> Box:
    return Box((0, 0, 0), tuple(int(s) for s in shape))


def box_for_ranges(lo_zyx, hi_zyx, volume_shape) -> Box:
    """The box [lo, hi) clamped to the volume, its faces open where the clamp did not reach the volume's."""
    lo = [max(0, int(v)) for v in lo_zyx]
    hi = [min(int(s), int(v)) for v, s in zip(hi_zyx, volume_shape)]
    faces = []
    for a, b, s in zip(lo, hi, volume_shape):
        faces += [a > 0, b < int(s)]
    return Box(tuple(lo), tuple(b - a for a, b in zip(lo, hi)), tuple(faces))


def _box_for(coords, pad, volume_shape) -> Box:
    """tiling.py:191-201: the smallest box holding every node's window plus ``pad`` (px, py, pz)."""
    c = np.asarray(coords, dtype=np.int64)
    lo = [int(c[:, k].min()) - pad[k] for k in (2, 1, 0)]
    hi = [int(c[:, k].max()) + pad[k] + 1 for k in (2, 1, 0)]
    return box_for_ranges(lo, hi, volume_shape)


# --------------------------------------------------------------------------- halo (tiling.py:141-175)
def tile_pad(p, half, disp=None, deformed: bool = False) -> tuple:
    """Voxels a box holds beyond a node centre, per axis (px, py, pz).  The reference side: the subset half-width,
    the gradient stencil and the presmoothing's reach.  The deformed side adds the displacement present in
    ``disp`` (measured, non-finite rows ignored), ``tile_disp_margin`` (0: the largest grid step), the subset's own
    stretch (``tile_strain_margin`` of the half-width), the search radius and the cubic sampling margin."""
    pad = [int(h) + REF_STENCIL_PAD for h in half]
    sigma = float(getattr(p, "prefilter_sigma", 0.0) or 0.0)
    if sigma > 0:
        pad = [q + int(4.0 * sigma + 0.5) for q in pad]
    if not deformed:
        return tuple(pad)
    strain = float(getattr(p, "tile_strain_margin", 0.25) or 0.0)
    radius = np.broadcast_to(np.asarray(getattr(p, "search_radius", 0), dtype=np.int64), (3,))
    margin = int(getattr(p, "tile_disp_margin", 0) or 0)
    if margin <= 0:
        margin = int(max(np.broadcast_to(np.asarray(p.winstepsize, dtype=np.int64), (3,))))
    moved = [0, 0, 0]
    if disp is not None and np.size(disp):
        d = np.abs(np.asarray(disp, dtype=np.float64))
        fin = d[np.isfinite(d).all(axis=1)] if d.ndim == 2 else d
        if fin.size:
            moved = [int(np.ceil(fin[:, k].max())) for k in range(3)]
    return tuple(int(q + moved[k] + margin + int(np.ceil(strain * h)) + int(radius[k]) + SAMPLE_PAD)
                 for k, (h, q) in enumerate(zip(half, pad)))


# --------------------------------------------------------------------------- plan (tiling.py:204-289)
@dataclass
class Tile:
    """One block of nodes (global indices, C order of the block) and its box; ``axes`` the block's lattice index
    ranges (iz, iy, ix) when the block is a whole sub-lattice."""

    nodes: np.ndarray
    box: Box
    axes: tuple | None = None


@dataclass
class TilePlan:
    tiles: list
    ref_pad: tuple
    def_pad: tuple
    fallback: str = ""

    def __len__(self) -> int:
        return len(self.tiles)

    def __iter__(self):
        return iter(self.tiles)

    @property
    def is_whole(self) -> bool:
        return len(self.tiles) == 1 and self.tiles[0].box.is_whole

    @property
    def max_voxels(self) -> int:
        return max((t.box.n_voxels for t in self.tiles), default=0)


def _blocks(n: int, count: int) -> list:
    count = max(1, min(int(count), int(n)))
    return [b for b in np.array_split(np.arange(n, dtype=np.int64), count) if b.size]


def plan_tiles(grid_shape, coords_xyz, volume_shape, p, half, disp=None, nodes=None, edge: int | None = None,
               pad: tuple | None = None) -> TilePlan:
    """Split the node lattice ``grid_shape`` (nz, ny, nx) into blocks whose boxes fit ``edge`` (default
    ``p.tile_local``) voxels per axis, as the reference's plan_tiles: each lattice axis split into near-equal
    contiguous blocks, as many as the node span over (edge - 2 halo) needs.  ``nodes`` restricts the plan (the
    escape retry); ``pad`` (px, py, pz) replaces the larger of the reference and deformed halos.  With the target
    at 0, or below one subset plus its halo, the plan is one whole-volume box."""
    volume_shape = tuple(int(s) for s in volume_shape)
    coords_xyz = np.asarray(coords_xyz, dtype=np.int64)
    n_total = coords_xyz.shape[0]
    index = np.arange(n_total, dtype=np.int64) if nodes is None else np.asarray(nodes, dtype=np.int64)
    ref_pad = tile_pad(p, half, deformed=False)
    def_pad = tile_pad(p, half, disp=disp, deformed=True)
    if pad is None:
        pad = tuple(max(r, d) for r, d in zip(ref_pad, def_pad))
    target = int(edge if edge is not None else getattr(p, "tile_local", 0) or 0)
    gz, gy, gx = (int(s) for s in grid_shape)
    full = index.size == n_total
    whole = TilePlan([Tile(index, whole_box(volume_shape), (np.arange(gz), np.arange(gy), np.arange(gx)) if full else None)],
                     ref_pad, def_pad)
    if target <= 0 or index.size == 0:
        return whole
    smallest = max(2 * q + 1 for q in pad)
    if smallest > target:
        whole.fallback = (f"tile_local={target} is smaller than one subset plus its halo ({smallest} voxels); "
                          "the local steps run on the whole volume")
        return whole
    if gz * gy * gx != n_total:
        whole.fallback = "the node grid is not a full lattice"
        return whole
    selected = np.zeros(n_total, dtype=bool)
    selected[index] = True
    counts = []
    for axis in range(3):  # z, y, x
        q = pad[2 - axis]
        room = target - 2 * q
        span = int(coords_xyz[:, 2 - axis].max() - coords_xyz[:, 2 - axis].min()) + 1
        counts.append(max(1, int(np.ceil(span / max(room, 1)))))
    lattice = np.arange(n_total, dtype=np.int64).reshape(gz, gy, gx)
    tiles = []
    for bz in _blocks(gz, counts[0]):
        for by in _blocks(gy, counts[1]):
            for bx in _blocks(gx, counts[2]):
                block = lattice[np.ix_(bz, by, bx)].ravel()
                keep = selected[block]
                if keep.sum() < MIN_TILE_NODES:
                    continue
                whole_block = bool(keep.all())
                block = block[keep]
                tiles.append(Tile(block, _box_for(coords_xyz[block], pad, volume_shape), (bz, by, bx) if whole_block else None))
    if not tiles:
        return whole
    covered = np.concatenate([t.nodes for t in tiles])
    if covered.size != index.size or not np.array_equal(np.sort(covered), np.sort(index)):
        whole.fallback = "the tile plan did not cover every node exactly once"
        return whole
    return TilePlan(tiles, ref_pad, def_pad)


def _quantised(pad) -> tuple:
    return tuple(int(-(-int(q) // PAD_QUANTUM) * PAD_QUANTUM) for q in pad)


def ncc_windows(coords_xyz, half, radius, shift, volume_shape) -> tuple:
    """Per node the voxel range [lo, hi) (z, y, x columns) an integer search reads: its template in f and its search
    window in g, the window clamped to the volume as the search clamps it (integer_search.py:376-386)."""
    c = np.asarray(coords_xyz, dtype=np.int64)
    s = np.zeros_like(c) if shift is None else np.asarray(shift, dtype=np.int64)
    lo, hi = [], []
    for k_xyz in (2, 1, 0):
        n = int(volume_shape[2 - k_xyz])
        h, r = int(half[k_xyz]), int(radius[k_xyz])
        w = 2 * h + 1 + 2 * r
        w0 = np.clip(c[:, k_xyz] + s[:, k_xyz] - h - r, 0, max(n - w, 0))
        lo.append(np.maximum(np.minimum(w0, c[:, k_xyz] - h), 0))
        hi.append(np.minimum(np.maximum(w0 + w, c[:, k_xyz] + h + 1), n))
    return np.stack(lo, axis=1), np.stack(hi, axis=1)


def plan_ncc_boxes(coords_xyz, half, radius, shift, volume_shape, edge: int) -> list:
    """Groups of nodes (positions in ``coords_xyz``) with boxes holding every read of their integer search: each
    axis's distinct node positions split into contiguous groups, as many as the node span over (edge - the
    widest read) needs; one group when ``edge`` is 0."""
    c = np.asarray(coords_xyz, dtype=np.int64)
    M = c.shape[0]
    if M == 0:
        return []
    lo, hi = ncc_windows(c, half, radius, shift, volume_shape)
    if edge <= 0:
        return [(np.arange(M), box_for_ranges(lo.min(axis=0), hi.max(axis=0), volume_shape))]
    labels = []
    for a_zyx, k_xyz in ((0, 2), (1, 1), (2, 0)):
        vals = np.unique(c[:, k_xyz])
        reach = int(np.max(np.maximum(c[:, k_xyz] - lo[:, a_zyx], hi[:, a_zyx] - 1 - c[:, k_xyz])))
        room = int(edge) - 2 * reach
        span = int(vals[-1] - vals[0]) + 1
        count = len(vals) if room <= 0 else max(1, int(np.ceil(span / room)))
        group_of_val = np.empty(len(vals), dtype=np.int64)
        for gi, part in enumerate(np.array_split(np.arange(len(vals)), max(1, min(count, len(vals))))):
            group_of_val[part] = gi
        labels.append(group_of_val[np.searchsorted(vals, c[:, k_xyz])])
    key = (labels[0] * (M + 1) + labels[1]) * (M + 1) + labels[2]
    out = []
    for k in np.unique(key):
        sel = np.flatnonzero(key == k)
        out.append((sel, box_for_ranges(lo[sel].min(axis=0), hi[sel].max(axis=0), volume_shape)))
    return out


# --------------------------------------------------------------------------- the frames in host memory
STAGING_SLOTS = 3  # pinned buffers in the ring: a crop is gathered into one while earlier ones are still copying
COPY_THREADS = max(1, min(16, os.cpu_count() or 1))  # host threads gathering one crop
PARALLEL_GATHER_BYTES = 8 << 20  # smaller crops are gathered by one thread

_TORCH_DTYPE = {np.dtype(np.float32): torch.float32, np.dtype(np.uint16): torch.uint16, np.dtype(np.uint8): torch.uint8}


class _Staging:
    """Host -> device copies of box crops: each crop is gathered from its (strided) host view into a pinned buffer by
    several threads, then copied on a stream of its own, so the copy of the next box overlaps the kernels of the
    current one.  The compute stream waits for each copy with an event; a pinned buffer is reused once the copy
    that read it has completed."""

    def __init__(self):
        self.stream = torch.cuda.Stream()
        self.slots: list = [(None, None)] * STAGING_SLOTS
        self.next = 0
        self.size = 0  # every slot grows to the largest crop seen, so a later pass allocates nothing
        self.pool = ThreadPoolExecutor(COPY_THREADS) if COPY_THREADS > 1 else None

    def _gather(self, dst: np.ndarray, src: np.ndarray) -> None:
        if self.pool is None or src.nbytes < PARALLEL_GATHER_BYTES or src.ndim == 0:
            np.copyto(dst, src)
            return
        axis = 0 if src.shape[0] >= COPY_THREADS or src.ndim == 1 else 1
        n = src.shape[axis]
        cuts = np.linspace(0, n, min(COPY_THREADS, n) + 1).astype(np.int64)

        def part(k):
            sl = (slice(None),) * axis + (slice(int(cuts[k]), int(cuts[k + 1])),)
            np.copyto(dst[sl], src[sl])

        list(self.pool.map(part, range(len(cuts) - 1)))

    def upload(self, a: np.ndarray) -> torch.Tensor:
        a = np.asarray(a)
        dt = _TORCH_DTYPE.get(a.dtype)
        if dt is None:
            raise TypeError(f"no staging copy for dtype {a.dtype}")
        k = self.next
        self.next = (k + 1) % len(self.slots)
        buf, done = self.slots[k]
        if done is not None:
            done.synchronize()  # the copy that last read this buffer has completed
        nbytes = max(int(a.nbytes), 1)
        self.size = max(self.size, nbytes)
        if buf is None or buf.numel() < nbytes:
            buf = None
            buf = torch.empty(self.size, dtype=torch.uint8, pin_memory=True)
        self._gather(buf[:nbytes].numpy().view(a.dtype)[: a.size].reshape(a.shape), a)
        pinned = buf[:nbytes].view(dt)[: a.size].view(a.shape)
        compute = torch.cuda.current_stream()
        with torch.cuda.stream(self.stream):
            dev = torch.empty(a.shape, dtype=dt, device="cuda")
            dev.copy_(pinned, non_blocking=True)
            done = torch.cuda.Event()
            done.record(self.stream)
        compute.wait_event(done)
        dev.record_stream(compute)
        self.slots[k] = (buf, done)
        return dev


_STAGING: dict = {}  # one ring per device, kept for the process: pinned buffers are slow to allocate


def _staging() -> _Staging:
    d = torch.cuda.current_device()
    if d not in _STAGING:
        _STAGING[d] = _Staging()
    return _STAGING[d]


def release_staging() -> None:
    """Free the pinned staging buffers of every device (the next tiled pass allocates them again)."""
    for st in _STAGING.values():
        for _, done in st.slots:
            if done is not None:
                done.synchronize()
    _STAGING.clear()


TILE_STREAMS = 2  # box solves alternate over this many streams, so one box's kernel tail overlaps the next box


def _tile_streams() -> list:
    d = torch.cuda.current_device()
    if d not in _TILE_STREAM_POOL:
        _TILE_STREAM_POOL[d] = [torch.cuda.Stream() for _ in range(TILE_STREAMS)]
    return _TILE_STREAM_POOL[d]


_TILE_STREAM_POOL: dict = {}


def _on_streams(items, fn) -> None:
    """``fn(item)`` for every item, alternating over the tile streams; each stream starts after the current
    stream's earlier work and the current stream waits for all of them at the end."""
    main = torch.cuda.current_stream()
    streams = _tile_streams()
    for st in streams:
        st.wait_stream(main)
    for i, it in enumerate(items):
        with torch.cuda.stream(streams[i % len(streams)]):
            fn(it)
    for st in streams:
        main.wait_stream(st)


def slab_ranges(shape, slab_voxels: int, step: int = 1) -> list:
    """z ranges [z0, z1) covering a volume of ``shape``, each of at most ``slab_voxels`` voxels where a multiple of
    ``step`` planes allows it and every one but the last a multiple of ``step`` planes."""
    nz, ny, nx = (int(s) for s in shape)
    t = max(step, (max(1, int(slab_voxels) // (ny * nx)) // step) * step)
    return [(z0, min(nz, z0 + t)) for z0 in range(0, nz, t)]


def _host_volume(a) -> np.ndarray:
    a = a.detach().cpu().numpy() if isinstance(a, torch.Tensor) else np.asarray(a)
    if a.ndim != 3:
        raise ValueError(f"expected a 3-D volume, got shape {a.shape}")
    if a.dtype not in (np.float32, np.uint16):
        a = a.astype(np.float32)
    return a


@dataclass
class FrameStats:
    """Whole-volume FP64 moments about ``pilot`` (device, 2 doubles) of ``n`` voxels."""

    sums: torch.Tensor
    n: int
    pilot: float


class HostFrames:
    """The reference and deformed frames (raw float32 / uint16) and masks in host memory, served to the device one
    box at a time in the forms the pass reads: normalised (and presmoothed) f, its gradients and the mask; the NCC
    input g (deformed mask -> 0); the interpolated g (B-spline coefficients with a B-spline, deformed mask -> NaN)
    and its overlapping-quad copy.  Boxes are kept on the device while ``cache_bytes`` allows (the first ones of
    a stage, so a cycle of boxes larger than the cache still hits on the kept ones)."""

    def __init__(self, f, g, p, mask=None, g_mask=None, normalize: bool = True, cache_bytes: int | None = None,
                 slab_voxels: int = SLAB_VOXELS):
        self.f = _host_volume(f)
        self.g = _host_volume(g)
        if self.f.shape != self.g.shape:
            raise ValueError("f and g must have the same shape")
        self.shape = tuple(int(s) for s in self.f.shape)
        self.mask = None if mask is None else np.asarray(mask)
        self.g_mask = None if g_mask is None else np.asarray(g_mask)
        for m in (self.mask, self.g_mask):
            if m is not None and tuple(m.shape) != self.shape:
                raise ValueError("mask shape differs from the volume shape")
        self.p = p
        self.mode = K.INTERP_MODE_BY_NAME[p.interp_method]
        self.sigma = float(p.prefilter_sigma or 0.0)
        self.smooth_reach = int(4.0 * self.sigma + 0.5) if self.sigma > 0 else 0
        self.slab_voxels = int(slab_voxels)
        self.normalize = normalize
        self.bytes_uploaded = 0
        self.boxes_loaded = 0
        self.cache_hits = 0
        if cache_bytes is None:
            free, _ = torch.cuda.mem_get_info()
            cache_bytes = free // 2
        self.cache_bytes = int(cache_bytes)
        self._cache: dict = {}
        self._cached = 0
        self.stats = {}
        if normalize:
            for name in ("f", "g"):
                self.stats[name] = self._moments(getattr(self, name))

    # ---- host -> device
    def _upload(self, a: np.ndarray) -> torch.Tensor:
        """A device copy of the host array (or strided view) ``a``, through the pinned staging ring."""
        self.bytes_uploaded += a.nbytes
        return _staging().upload(a)

    def slabs(self, step: int = 1):
        return slab_ranges(self.shape, self.slab_voxels, step)

    def _moments(self, vol: np.ndarray) -> FrameStats:
        nz, ny, nx = self.shape
        pilot = float(vol[nz // 2, ny // 2, nx // 2])  # the reference's pilot: the centre voxel (io/volume_ops.py:91)
        sums = torch.zeros(2, dtype=torch.float64, device="cuda")
        for z0, z1 in self.slabs():
            K.volume_moments(self._upload(vol[z0:z1]), pilot, sums)
        return FrameStats(sums, int(vol.size), pilot)

    def _normalised(self, name: str, box: Box) -> torch.Tensor:
        raw = self._upload(box.view(getattr(self, name)))
        if not self.normalize:
            return raw.float().contiguous()
        st = self.stats[name]
        return K.normalize_sums(raw, st.sums, st.n, st.pilot)

    def _frame(self, name: str, box: Box) -> torch.Tensor:
        """Normalised (and presmoothed) frame ``name`` over ``box``: the presmoothing runs on the box grown by its
        reach."""
        if self.smooth_reach == 0:
            return self._normalised(name, box)
        big, inner = box.grown((self.smooth_reach,) * 3, self.shape)
        v = K.gaussian_presmooth(self._normalised(name, big), self.sigma)
        return v[inner].contiguous()

    def _mask_of(self, m, box: Box):
        return None if m is None else self._upload((box.crop(m) != 0).astype(np.uint8))

    # ---- what the stages read
    def _cache_put(self, key, vols: dict):
        nbytes = sum(t.numel() * t.element_size() for t in vols.values() if isinstance(t, torch.Tensor))
        if self._cached + nbytes <= self.cache_bytes:
            self._cache[key] = vols
            self._cached += nbytes

    def _hit(self, v: dict) -> dict:
        """A kept box, read by the current stream (which may not be the one that built it)."""
        self.cache_hits += 1
        cur = torch.cuda.current_stream()
        for t in v.values():
            if isinstance(t, torch.Tensor):
                t.record_stream(cur)
        return v

    def clear_cache(self):
        self._cache.clear()
        self._cached = 0

    def ncc_volumes(self, box: Box) -> tuple:
        """(f, g) of the integer search over ``box``: normalised, presmoothed, the deformed mask's voxels of g -> 0."""
        self.boxes_loaded += 1
        return self._frame("f", box), self.ncc_g(box)

    def ncc_g(self, box: Box) -> torch.Tensor:
        """The NCC input g over ``box``."""
        g = self._frame("g", box)
        if self.g_mask is not None:
            K.mask_fill(g, self._mask_of(self.g_mask, box), 0.0)
        return g

    def reference_volumes(self, box: Box) -> dict:
        """f, its gradients and the mask over ``box`` (the precompute)."""
        v = self._cache.get(("local", box.origin, box.shape))
        if v is not None:
            return self._hit(v)
        self.boxes_loaded += 1
        f = self._frame("f", box)
        gx, gy, gz = K.gradients(f)
        return {"f": f, "gx": gx, "gy": gy, "gz": gz, "m": self._mask_of(self.mask, box)}

    def local_volumes(self, box: Box, quads: bool) -> dict:
        """Everything the IC-GN reads over ``box``: the reference volumes plus the interpolated g (B-spline
        coefficients from the box grown by the prefilter's reach) and, with ``quads``, its overlapping quads.  Only
        these are kept between stages: the 12-DOF step and every ADMM step read them again."""
        key = ("local", box.origin, box.shape)
        v = self._cache.get(key)
        if v is not None and (v["g4"] is not None or not quads):
            return self._hit(v)
        v = dict(self.reference_volumes(box))
        if self.mode == 2:  # B-spline: prefilter the box grown by the filter's reach, keep the box
            big, inner = box.grown((BSPLINE_REACH,) * 3, self.shape)
            g_prep = K.bspline_prefilter(self._frame("g", big))[inner].contiguous()
        else:
            g_prep = self._frame("g", box)
        if self.g_mask is not None:
            K.mask_fill(g_prep, self._mask_of(self.g_mask, box), float("nan"))
        v["g"] = g_prep
        v["g4"] = K.make_quads(g_prep) if quads else None
        self._cache_put(key, v)
        return v

    # ---- whole-volume sweeps
    def block_means(self, factors) -> dict:
        """{factor: (f, g) block means on the device}: the whole pair swept slab by slab, each slab a whole number
        of blocks of every factor (the trailing voxels of each axis dropped, as block_downsample does)."""
        factors = sorted({int(k) for k in factors if int(k) > 1})
        if not factors:
            return {}
        step = math.lcm(*factors)
        nz = self.shape[0]
        parts = {k: ([], []) for k in factors}
        for z0, z1 in self.slabs(step):
            box = Box((z0, 0, 0), (z1 - z0,) + self.shape[1:], (z0 > 0, z1 < nz, False, False, False, False))
            f, g = self._frame("f", box), self.ncc_g(box)
            self.boxes_loaded += 1
            for k in factors:
                if (z1 - z0) // k > 0:
                    parts[k][0].append(K.block_downsample(f, k))
                    parts[k][1].append(K.block_downsample(g, k))
        return {k: (torch.cat(a, 0).contiguous(), torch.cat(b, 0).contiguous()) for k, (a, b) in parts.items() if a}

    def f_std(self) -> float:
        """Population standard deviation of the normalised (presmoothed) f, FP64 moments about its centre voxel,
        swept slab by slab."""
        nz, ny, nx = self.shape
        pilot = float(self._frame("f", Box((nz // 2, ny // 2, nx // 2), (1, 1, 1)))[0, 0, 0].item())
        sums = torch.zeros(2, dtype=torch.float64, device="cuda")
        for z0, z1 in self.slabs():
            K.volume_moments(self._frame("f", Box((z0, 0, 0), (z1 - z0,) + self.shape[1:], (z0 > 0, z1 < nz) + (False,) * 4)),
                             pilot, sums)
        ts, tq = (float(v) for v in sums.cpu().numpy())
        n = float(np.prod(self.shape))
        ms = ts / n
        return math.sqrt(max(tq / n - ms * ms, 0.0))


# --------------------------------------------------------------------------- box-wise searches and solves
def _gather(t, idx):
    return None if t is None else t[idx]


@dataclass
class TileRecord:
    """Boxes per stage: count, the largest box's voxels, and the nodes retried with a wider halo."""

    stages: dict = field(default_factory=dict)

    def add(self, stage: str, boxes: list, retried: int = 0):
        s = self.stages.setdefault(stage, {"calls": 0, "boxes": 0, "max_voxels": 0, "retried": 0})
        s["calls"] += 1
        s["boxes"] += len(boxes)
        s["max_voxels"] = max([s["max_voxels"]] + [b.n_voxels for b in boxes])
        s["retried"] += int(retried)


class _Shape:
    """A stand-in for a volume that only gives its shape (the whole-volume checks of the integer search)."""

    def __init__(self, shape):
        self.shape = tuple(shape)


def _box_search(frames: HostFrames, edge: int, record: TileRecord):
    """search_fn of the integer search: the nodes grouped into boxes that hold their template and clamped window,
    each group searched on its box's (f, g) with box-frame coordinates."""

    def search(c, half, radius, sh, eng):
        c_np = c.cpu().numpy()
        sh_np = None if sh is None else sh.cpu().numpy()
        M = c_np.shape[0]
        out = {"disp": torch.full((M, 3), float("nan"), dtype=torch.float64, device="cuda"),
               "cc": torch.full((M,), float("nan"), dtype=torch.float64, device="cuda"),
               "pce": torch.full((M,), float("nan"), dtype=torch.float64, device="cuda"),
               "clipped": torch.zeros(M, dtype=torch.uint8, device="cuda"), "ok": torch.zeros(M, dtype=torch.uint8, device="cuda")}
        groups = plan_ncc_boxes(c_np, half, radius, sh_np, frames.shape, edge)
        record.add("ncc", [b for _, b in groups])
        for sel, box in groups:
            fb, gb = frames.ncc_volumes(box)
            idx = torch.from_numpy(sel).cuda()
            cb = torch.from_numpy(box.shift(c_np[sel])).cuda()
            res = K.ncc_search(fb, gb, cb, half, radius, None if sh is None else sh[idx].contiguous(), eng)
            for k in out:
                out[k][idx] = res[k].to(out[k].dtype)
        return out

    return search


def _morton_rank(mesh) -> np.ndarray:
    order = mesh.order().cpu().numpy()
    rank = np.empty(mesh.n, dtype=np.int64)
    rank[order] = np.arange(mesh.n)
    return rank


MARGIN_LO, MARGIN_HI = 1.0, 3.0  # interp_kernels.interp_margin_ok: a sample needs 1 voxel below and 3 above it
LEFT_VOLUME_TOL = 1e-9  # voxels: far above the FP64 difference between box-local and volume positions


def left_volume(P, coords_xyz, half, stride, volume_shape) -> np.ndarray:
    """Per node (rows of ``P`` (M, 12), the iterate a solve stopped at, and ``coords_xyz`` (M, 3) in the volume's
    frame) whether a corner voxel of its warped subset lies outside the volume's sampling margin by more than
    ``LEFT_VOLUME_TOL``.  The reference's sampler fails a node as soon as one unmasked warped voxel leaves that
    margin (numba_kernels.py:563-576); for a node with no mask whose subset lies inside the volume every voxel is
    visited and the warp is affine, so the corners decide: such a node fails at the same iterate on the whole
    volume and needs no retry in a wider box."""
    P = np.asarray(P, dtype=np.float64).reshape(-1, 12)
    c = np.asarray(coords_xyz, dtype=np.float64).reshape(-1, 3)
    hi = [-int(h) + ((2 * int(h)) // int(stride)) * int(stride) for h in half]
    corners = np.array([[dx, dy, dz] for dz in (-half[2], hi[2]) for dy in (-half[1], hi[1]) for dx in (-half[0], hi[0])],
                       dtype=np.float64)  # (8, 3) offsets [x, y, z]
    A = P[:, :9].reshape(-1, 3, 3) + np.eye(3)[None]
    w = np.einsum("nij,kj->nki", A, corners) + (c + P[:, 9:12])[:, None, :]  # (M, 8, 3) warped [x, y, z]
    n_xyz = np.array(volume_shape[::-1], dtype=np.float64)
    out = (w < MARGIN_LO - LEFT_VOLUME_TOL) | (w > n_xyz - MARGIN_HI + LEFT_VOLUME_TOL)
    return out.any(axis=(1, 2))


def _solve_tiles(plan_fn, solve_fn, status_out, stage: str, record: TileRecord, base_pad, extra_pad, left_fn=None):
    """Run ``solve_fn(tile)`` over the tiles of ``plan_fn(nodes, pad)``; nodes whose status says they left an open
    face of their box are planned again with the halo widened by ``extra_pad`` per retry (the reference retries them
    on the whole volume, local_icgn.py:448-459).  ``left_fn(nodes)`` marks those of them whose last iterate left the
    volume itself: they would fail on the whole volume too, and are not retried."""
    plan = plan_fn(None, base_pad)
    record.add(stage, [t.box for t in plan])
    open_face = np.zeros(status_out.shape[0], dtype=bool)
    _on_streams(plan.tiles, solve_fn)
    for t in plan:
        open_face[t.nodes] = t.box.has_open_face
    pad = base_pad
    retried = 0
    for _ in range(ESCAPE_RETRIES):
        st = status_out.cpu().numpy()
        escaped = np.flatnonzero((st == STATUS_OUT_OF_BOUNDS) & open_face)
        if escaped.size and left_fn is not None:
            escaped = escaped[~left_fn(escaped)]
        if escaped.size == 0:
            break
        retried += escaped.size
        pad = tuple(q + e for q, e in zip(pad, extra_pad))
        plan = plan_fn(escaped, pad)
        record.add(stage + "_retry", [t.box for t in plan], escaped.size)
        open_face[:] = False
        _on_streams(plan.tiles, solve_fn)
        for t in plan:
            open_face[t.nodes] = t.box.has_open_face
    return retried


def _launch_shape(p, ndof: int, mode: int, mesh, masked: bool, plan: TilePlan, run_tile) -> tuple:
    """(threads, brick_floats) of the tiled IC-GN launches: the caller's, else the autotuner's choice for this kernel
    and subset (the cache key of the whole-volume pass, so both passes share it), timed on an evenly spread sample
    of the nodes of the plan's largest tile."""
    if p.variant != K.BATCHED or p.threads != 0 or not p.autotune or p.node_winsize is not None:
        return p.threads, p.brick_floats
    k = autotune.key(ndof, mode, True, mesh.half, p.subset_stride, masked, mesh.n)
    t = max(plan.tiles, key=lambda t_: len(t_.nodes))
    sub = t.nodes[autotune.sample_index(len(t.nodes)).cpu().numpy()]
    return autotune.tune(k, lambda th, br: run_tile(t, sub, (th, br)))


def run_pass_tiled(f, g, p, mask=None, g_mask=None, normalize: bool = True, edge: int | None = None,
                   tracer: PL.Tracer | None = None, cache_bytes: int | None = None, slab_voxels: int = SLAB_VOXELS,
                   frames: HostFrames | None = None, previous: torch.Tensor | None = None) -> PL.PassResult:
    """One AL-DVC pass (core/pipeline.py:255-366) with every voxel-reading step run box by box from host memory.

    ``f``, ``g``: host volumes (NumPy arrays or memory maps, float32 or uint16; CPU tensors are accepted);
    ``mask`` / ``g_mask``: host reference / deformed-frame masks; ``edge``: the box edge target in voxels
    (default ``p.tile_local``; 0 runs one whole-volume box).  ``cache_bytes`` bounds the device memory kept for
    boxes between stages (default half the free memory).  The result is ``run_pass``'s on the same frames, with
    ``result.tiles`` recording the boxes of every stage and ``result.frames`` the host frames (bytes uploaded,
    boxes loaded, cache hits).  The ADMM loop runs eagerly (no graph capture: every step streams boxes).
    ``previous``: the last frame's field against the same reference, for ``init_guess_method="previous"``."""
    tr = tracer if tracer is not None else PL.Tracer(sync=False)
    tr.start()
    errs = K.ErrorWords()
    own_frames = frames is None
    if own_frames:
        frames = HostFrames(f, g, p, mask, g_mask, normalize, cache_bytes, slab_voxels)
    edge = int(p.tile_local if edge is None else edge)
    record = TileRecord()
    mode = frames.mode
    mesh = PL.Mesh(frames.shape, p)
    coords_np = mesh.coords_np
    half = mesh.half
    tr.mark("preprocess")

    # ---------------- precompute, box by box (local_icgn.py:239-330)
    node_half = None
    if p.node_winsize is not None:
        ws = np.asarray(p.node_winsize(coords_np), dtype=np.int64).reshape(-1, 3)
        hs = ws // 2
        if (hs > np.asarray(half)[None, :]).any():
            raise ValueError("node_winsize exceeds winsize")
        node_half = torch.from_numpy(hs.astype(np.int32)).cuda()
    N = mesh.n
    H = torch.zeros((N, 12, 12), dtype=torch.float64, device="cuda")
    L = torch.zeros((N, 12, 12), dtype=torch.float64, device="cuda")
    meanf = torch.zeros(N, dtype=torch.float64, device="cuda")
    bottomf = torch.ones(N, dtype=torch.float64, device="cuda")
    n_valid = torch.zeros(N, dtype=torch.int64, device="cuda")
    valid = torch.zeros(N, dtype=torch.uint8, device="cuda")
    pre_plan = plan_tiles(mesh.grid_shape, coords_np, frames.shape, p, half, edge=edge)
    record.add("precompute", [t.box for t in pre_plan])
    forms = set()

    def precompute_tile(t):
        v = frames.reference_volumes(t.box)
        bz, by, bx = t.box.shape
        idx = torch.from_numpy(t.nodes).cuda()
        if (t.axes is not None and node_half is None and p.subset_stride == 1 and p.variant == K.BATCHED and bx <= 8192
                and by <= 65535):
            iz, iy, ix = t.axes
            z0, y0, x0 = t.box.origin
            out = K.precompute_grid(mesh.axes[0][ix] - x0, mesh.axes[1][iy] - y0, mesh.axes[2][iz] - z0, half, v["f"], v["gx"],
                                    v["gy"], v["gz"], p.min_valid_ratio, p.hessian_cond_max, v["m"])
            forms.add("grid")
        else:
            cb = torch.from_numpy(t.box.shift(coords_np[t.nodes])).cuda()
            out = K.precompute(cb, half, v["f"], v["gx"], v["gy"], v["gz"], v["m"], p.min_valid_ratio, p.hessian_cond_max,
                               p.subset_stride, None, None, _gather(node_half, idx))
            forms.add("per_node")
        for dst, src in zip((H, L, meanf, bottomf, n_valid, valid), out):
            dst[idx] = src

    _on_streams(pre_plan.tiles, precompute_tile)
    valid_b = valid != 0
    centre_ok = None
    if frames.mask is not None:
        c = coords_np
        centre_ok = torch.from_numpy(frames.mask[c[:, 2], c[:, 1], c[:, 0]] != 0).cuda()
    valid_b, elem_active = PL.node_validity(mesh, p, node_half, valid_b, centre_ok, n_valid)
    valid_u8 = valid_b.to(torch.uint8).contiguous()
    tr.mark("precompute")

    # ---------------- section 3: initial guess, box-wise searches
    shape_only = _Shape(frames.shape)
    search_fn = _box_search(frames, edge, record)
    levels = None
    level_volumes = None
    shift_fn = None
    if p.init_guess_method != "zero":
        factors = []
        if p.global_shift:
            factors.append(max(1, int(math.ceil(max(frames.shape) / 128))))
        pyramid = p.init_guess_method in ("pyramid", "previous")
        if pyramid:
            factors += [2**lv for lv in range(1, (p.pyramid_levels if p.pyramid_levels > 0 else 3) + 1)]
        means = frames.block_means(factors)
        if p.global_shift:
            fac = factors[0]
            shift_fn = lambda: IS.phase_correlation_shift_device(shape_only, shape_only,  # noqa: E731
                                                                 downsample=lambda k: means[k] if k > 1 else None)
            if fac == 1:  # a volume of at most 128 voxels per axis: the full-resolution pair
                box = whole_box(frames.shape)
                shift_fn = lambda: IS.phase_correlation_shift_device(*frames.ncc_volumes(box))  # noqa: E731
        if pyramid:
            level_volumes = lambda k: means[k]  # noqa: E731
            subset0 = p.init_subset if p.init_subset is not None else tuple(min(int(w), 16) for w in p.winsize)
            levels = p.pyramid_levels
            if levels <= 0:
                levels = IS.auto_pyramid_levels(frames.shape, subset0, tuple(int(r) for r in p.search_radius),
                                                std0=frames.f_std(), downsample=lambda k: means[k][0])
    ncc_calls: list = []
    U0, init_info = PL.initial_guess(p, mesh, shape_only, shape_only, valid_b, ncc_calls, errs, previous=previous, shift_fn=shift_fn,
                                     search_fn=search_fn, level_volumes=level_volumes, levels=levels)
    tr.mark("init_guess")

    # ---------------- section 4: local 12-DOF IC-GN, box by box
    quads = mode != 0 and p.variant == K.BATCHED and p.icgn_quads
    rank = _morton_rank(mesh) if (p.variant == K.BATCHED and p.icgn_node_order == "morton") else None
    P0 = torch.zeros((N, 12), dtype=torch.float64, device="cuda")
    P0[:, 9:] = U0
    P = torch.zeros((N, 12), dtype=torch.float64, device="cuda")
    n_iter = torch.zeros(N, dtype=torch.int32, device="cuda")
    status = torch.zeros(N, dtype=torch.int8, device="cuda")
    zncc = torch.zeros(N, dtype=torch.float64, device="cuda")
    margin = int(p.tile_disp_margin) if p.tile_disp_margin > 0 else int(max(np.broadcast_to(np.asarray(p.winstepsize), (3,))))
    extra = tuple(int(h) + margin for h in half)

    nz_, ny_, nx_ = frames.shape
    inside = ((coords_np[:, 0] - half[0] >= 0) & (coords_np[:, 0] + half[0] < nx_) & (coords_np[:, 1] - half[1] >= 0)
              & (coords_np[:, 1] + half[1] < ny_) & (coords_np[:, 2] - half[2] >= 0) & (coords_np[:, 2] + half[2] < nz_))

    def left_of(P_of):
        """The retry filter of a local step: with no reference mask and one subset shape, the out-of-bounds nodes
        whose subset lies inside the volume and whose last iterate (``P_of(index tensor)``, (M, 12)) left it."""
        if frames.mask is not None or node_half is not None:
            return None

        def left(nodes):
            out = np.zeros(len(nodes), dtype=bool)
            keep = inside[nodes]
            sel = nodes[keep]
            if sel.size:
                Pn = P_of(torch.from_numpy(sel).cuda()).cpu().numpy()
                out[keep] = left_volume(Pn, coords_np[sel], half, p.subset_stride, frames.shape)
            return out

        return left

    def order_of(nodes):
        if rank is None:
            return None
        return torch.from_numpy(np.argsort(rank[nodes], kind="stable").astype(np.int32)).cuda()

    def plan_local(disp):
        def plan_fn(nodes, pad):
            return plan_tiles(mesh.grid_shape, coords_np, frames.shape, p, half, disp=disp, nodes=nodes, edge=edge, pad=pad)
        pads = plan_tiles(mesh.grid_shape, coords_np, frames.shape, p, half, disp=disp, edge=0)
        return plan_fn, _quantised(tuple(max(a, b) for a, b in zip(pads.ref_pad, pads.def_pad)))

    shapes = {}

    def icgn12_tile(t, sub=None, shape=None):
        """Solve tile ``t``; with ``sub`` (some of its nodes) and ``shape`` only time a launch shape (no result kept)."""
        nodes = t.nodes if sub is None else sub
        th_, br_ = shapes[12] if shape is None else shape
        v = frames.local_volumes(t.box, quads)
        idx = torch.from_numpy(nodes).cuda()
        cb = torch.from_numpy(t.box.shift(coords_np[nodes])).cuda()
        res = K.icgn12(cb, P0[idx], half, v["f"], v["gx"], v["gy"], v["gz"], v["m"], v["g"], mode, L[idx], meanf[idx], valid_u8[idx],
                       p.icgn_tol, p.icgn_dp_tol, p.icgn_max_iter, p.icgn_patience, p.subset_stride, None, None, 0.0,
                       p.icgn_predictive_stop, None, None, p.variant, th_, br_, node_half=_gather(node_half, idx), g4=v["g4"],
                       sweep_rows=p.icgn_sweep_rows, node_order=order_of(nodes), errs=errs if sub is None else None)
        if sub is None:
            for dst, src in zip((P, n_iter, status, zncc), res):
                dst[idx] = src.to(dst.dtype)

    plan_fn, pad0 = plan_local(U0.cpu().numpy())
    shapes[12] = _launch_shape(p, 12, mode, mesh, frames.mask is not None, plan_fn(None, pad0), icgn12_tile)
    _solve_tiles(plan_fn, icgn12_tile, status, "icgn12", record, pad0, extra, left_of(lambda idx: P[idx]))
    bad = status != PL.STATUS_CONVERGED
    flag = PL._median_flags(P[:, 9:].contiguous(), ~bad, mesh.grid_shape, p.local_outlier_threshold, errs)
    bad = bad | flag
    UF, all_bad = PL._fill(P, bad, mesh.grid_shape, errs)
    if bool(all_bad.item()):
        UF.zero_()
    U1 = UF[:, 9:].contiguous()
    F1 = UF[:, :9].contiguous()
    tr.mark("local_icgn")

    result = PL.PassResult(U=U1, F=F1.reshape(-1, 3, 3), status=status, zncc=zncc, n_iter=n_iter, coords=mesh.coords,
                           grid_shape=mesh.grid_shape, valid=valid_b, U_local=U1.clone(), U0=U0, P_local=P, status_local=status,
                           n_iter_local=n_iter)
    result.F_local = F1.reshape(-1, 3, 3).clone()
    result.outlier = bad & (status == PL.STATUS_CONVERGED)
    result.tracer = tr
    result.ncc_calls = ncc_calls
    result.init_info = init_info
    result.precompute_form = "grid" if forms == {"grid"} else ("per_node" if forms == {"per_node"} else "mixed")
    result.node_half = node_half
    result.icgn3_iters = []
    result.tiles = record
    result.frames = frames
    # the reference quantities a frame series needs (uncertainty, strain): Hessians, node statistics, grid
    result.H, result.n_valid, result.bottomf = H, n_valid, bottomf
    result.elem_active, result.mesh = elem_active, mesh
    if not p.use_global_step:
        errs.check()
        if own_frames:
            frames.clear_cache()
        return result

    # ---------------- sections 5-6: ADMM with the 3-DOF step box by box
    beta = p.beta
    result.beta_sweep = None
    if beta is None:
        exclude = bad.clone()
        exclude[torch.from_numpy(surface_nodes(mesh.grid_shape)).cuda()] = True
        beta, result.beta_sweep = BT.auto_tune_beta_device(mesh.grid_shape, mesh.spacing, elem_active, p.mu, p.alpha, U1, F1, exclude,
                                                           p.winstepsize, p.beta_range, p.beta_criterion, p.pcg_tol, p.pcg_max_iter,
                                                           p.gauss_pt_order)
    result.beta = beta
    n_full = float(np.prod([(2 * h) // p.subset_stride + 1 for h in half]))
    global_step = PL.make_global_step(mesh, p, elem_active, beta, errs)

    def icgn3_all(U2_, F2_, v_):
        U = torch.zeros((N, 3), dtype=torch.float64, device="cuda")
        it = torch.zeros(N, dtype=torch.int32, device="cuda")
        st = torch.zeros(N, dtype=torch.int8, device="cuda")
        zc = torch.zeros(N, dtype=torch.float64, device="cuda")

        def tile3(t, sub=None, shape=None):
            nodes = t.nodes if sub is None else sub
            th_, br_ = shapes[3] if shape is None else shape
            v = frames.local_volumes(t.box, quads)
            idx = torch.from_numpy(nodes).cuda()
            cb = torch.from_numpy(t.box.shift(coords_np[nodes])).cuda()
            res = K.icgn3(cb, U2_[idx], F2_[idx], v_[idx], half, v["f"], v["gx"], v["gy"], v["gz"], v["m"], v["g"], mode, H[idx],
                          meanf[idx], bottomf[idx], valid_u8[idx], p.mu, p.icgn_tol, p.icgn_dp_tol, p.icgn_max_iter, p.icgn_patience,
                          p.subset_stride, n_full, 0.0, p.icgn_predictive_stop, None, None, p.variant, th_, br_,
                          node_half=_gather(node_half, idx), g4=v["g4"], sweep_rows=p.icgn_sweep_rows, node_order=order_of(nodes),
                          errs=errs if sub is None else None)
            if sub is None:
                for dst, src in zip((U, it, st, zc), res):
                    dst[idx] = src.to(dst.dtype)

        # subpb1_solver.py:34: the halo follows the displacement the 3-DOF step starts from, U_hat + vdual
        plan_fn3, pad3 = plan_local((U2_ + v_).cpu().numpy())
        if 3 not in shapes:
            shapes[3] = _launch_shape(p, 3, mode, mesh, frames.mask is not None, plan_fn3(None, pad3), tile3)
        _solve_tiles(plan_fn3, tile3, st, "icgn3", record, pad3, extra, left_of(lambda idx: torch.cat([F2_[idx], U[idx]], 1)))
        return U, it, st, zc

    W = torch.zeros((N, 9), dtype=torch.float64, device="cuda")
    v = torch.zeros((N, 3), dtype=torch.float64, device="cuda")
    U2, F2 = global_step(U1, F1, W, v)
    W = F2 - F1
    v = U2 - U1
    steps = 1
    st_last, zc_last, it_last = status, zncc, n_iter
    U1_prev = U1
    for step in range(2, p.admm_max_iter + 1):
        steps = step
        U, it_last, st_last, zc_last = icgn3_all(U2, F2, v)
        result.icgn3_iters.append(it_last)
        bad3 = st_last != PL.STATUS_CONVERGED
        bad3 = bad3 | PL._median_flags(U, ~bad3, mesh.grid_shape, p.local_outlier_threshold, errs)
        result.outlier = bad3 & (st_last == PL.STATUS_CONVERGED)
        U1n = torch.where(bad3[:, None], U2, U)
        F1n = F2
        U2n, F2n = global_step(U1n, F1n, W, v)
        if p.dual_update == "accumulate":
            W = W + (F2n - F1n)
            v = v + (U2n - U1n)
        else:
            W = F2n - F1n
            v = U2n - U1n
        du_g = PL._rms(U2n - U2)
        du_l = PL._rms(U1n - U1_prev)
        U1_prev = U1n
        U1, U2, F2 = U1n, U2n, F2n
        if p.admm_early_stop and (float(du_g.item()) < p.admm_tol or float(du_l.item()) < p.admm_tol):
            break
    errs.check()
    if own_frames:
        frames.clear_cache()  # the result keeps the frames' record, not their boxes
    tr.mark("admm")
    result.U = U2
    result.F = F2.reshape(-1, 3, 3)
    result.status, result.zncc, result.n_iter = st_last, zc_last, it_last
    result.admm_steps = steps
    return result
