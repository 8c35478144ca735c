"""A series of frames through the device pass: pyALDVC's run_aldvc frame loop (core/pipeline.py:82-452) and its
cumulative displacements (:455-491 _compose_cumulative), with the reference schedule of core/data_structures.py:
172-215 (FrameSchedule).

Frame k (k >= 1) is solved against its reference frame ``schedule.parent(k)``:

- a reference is prepared once (normalisation, gradients, node grid, precompute, node validity: the pipeline's
  ``prepare_reference``) and kept for later frames, at most ``REF_CACHE`` references at a time (pipeline.py:60,
  189-228);
- ``init_guess_method="previous"`` starts frame k from the last frame's field when that frame used the same
  reference (pipeline.py:266), else from the pyramid;
- a tuned beta is tuned once per reference and reused by its later frames (pipeline.py:291-296);
- the material points that started at the frame-0 nodes are tracked through each frame's reference chain: frame
  k's displacement grid is interpolated (cubic spline or trilinear, ``aldvc_grid_interp``) at the positions the
  parent frame's points have reached.

The frames may be host arrays (NumPy or CPU tensors, copied through pinned staging on a stream of their own, so
that frame k + 1 is on its way to the device while frame k is solved) or CUDA tensors.
"""

from __future__ import annotations

import copy
import threading
import time
from collections import OrderedDict
from concurrent.futures import ThreadPoolExecutor
from dataclasses import dataclass, field

import numpy as np
import torch

from . import kernels as K
from . import pipeline as PL
from . import uncertainty as UN
from .mesh import build_grid_axes, grid_coords

REF_CACHE = 2  # prepared references kept at a time (core/pipeline.py:60)


@dataclass(frozen=True)
class FrameSchedule:
    """The reference frame of every deformed frame: ``ref_indices[i]`` is the reference of frame i + 1, at most i
    (no frame references a later one)."""

    ref_indices: tuple

    def __post_init__(self):
        for i, r in enumerate(self.ref_indices):
            if not isinstance(r, (int, np.integer)):
                raise TypeError(f"ref_indices[{i}] must be int (got {type(r).__name__})")
            if r < 0:
                raise ValueError(f"ref_indices[{i}]={r} is negative")
            if r > i:
                raise ValueError(f"ref_indices[{i}]={r} references a future frame (must be <= {i})")

    @classmethod
    def from_mode(cls, mode: str, n_frames: int) -> "FrameSchedule":
        """"accumulative": every frame against frame 0; "incremental": every frame against the one before it."""
        if n_frames < 2:
            raise ValueError(f"n_frames must be >= 2 (got {n_frames})")
        if mode == "accumulative":
            return cls(tuple(0 for _ in range(n_frames - 1)))
        if mode == "incremental":
            return cls(tuple(range(n_frames - 1)))
        raise ValueError(f"Unknown reference mode '{mode}'. Use 'accumulative' or 'incremental'.")

    @classmethod
    def from_every_n(cls, n: int, n_frames: int) -> "FrameSchedule":
        """The reference moves on every ``n`` frames: frame d uses frame (d - 1) // n * n."""
        if n < 1:
            raise ValueError(f"n must be >= 1 (got {n})")
        if n_frames < 2:
            raise ValueError(f"n_frames must be >= 2 (got {n_frames})")
        return cls(tuple((d - 1) // n * n for d in range(1, n_frames)))

    def parent(self, frame: int) -> int:
        if frame < 1 or frame > len(self.ref_indices):
            raise IndexError(f"frame={frame} out of range [1, {len(self.ref_indices)}]")
        return int(self.ref_indices[frame - 1])


@dataclass
class StrainParams:
    """Strain of every frame (DVCPara strain_* fields, core/config.py:115-122): gradient method "plane_fit", "fd",
    "fem" or "direct" (frames against frame 0 use their own F), plane-fit half-width in nodes, strain measure,
    voxel size (x, y, z), Gaussian smoothing of the displacement and of the strain (in nodes), and whether nodes
    whose gradient stencil is incomplete are trimmed."""

    method: str = "plane_fit"
    halfwidth: tuple = (1, 1, 1)
    strain_type: str = "infinitesimal"
    voxel_size: tuple = (1.0, 1.0, 1.0)
    disp_smoothing: float = 0.0
    strain_smoothing: float = 0.0
    edge_trim: bool = True


@dataclass
class FrameResult:
    """One deformed frame (host arrays): the pass's displacements and gradients against reference ``ref_frame``,
    the local result and initial guess, final ZNCC and statuses, the outlier flags (converged, then rejected by
    the median test and replaced), the displacement accumulated from frame 0, the beta used and the ADMM steps."""

    U: np.ndarray
    F: np.ndarray
    ref_frame: int
    U_local: np.ndarray
    F_local: np.ndarray
    U0: np.ndarray
    zncc: np.ndarray
    status: np.ndarray
    outlier: np.ndarray
    valid: np.ndarray
    beta: float | None = None
    admm_steps: int = 0
    init_method: str = ""
    U_std: np.ndarray | None = None  # standard deviation of u, v, w (voxels) from the normal equations
    U_accum: np.ndarray | None = None
    strain: object = None  # strain.StrainResult of U_accum when run_series was given StrainParams
    seconds: float = 0.0


@dataclass
class SeriesResult:
    frames: list
    coords: np.ndarray  # (N, 3) [x, y, z] node positions in frame 0
    grid_shape: tuple
    axes: tuple  # node axes (x0, y0, z0), voxels
    schedule: FrameSchedule
    timings: dict = field(default_factory=dict)


class _Uploader:
    """Frames on the device, host ones copied ahead of use: ``prefetch(i)`` gathers frame i into pinned memory on a
    helper thread and copies it on a stream of its own; ``get(i)`` makes the current stream wait for that copy."""

    def __init__(self, volumes, masks):
        self.volumes = volumes
        self.masks = masks
        self.stream = torch.cuda.Stream()
        self.pool = ThreadPoolExecutor(1)
        self.lock = threading.Lock()
        self.pending: dict = {}
        self.h2d_bytes = 0

    def _stage(self, a):
        """(device tensor, event) of one host array copied on the upload stream; CUDA tensors pass through."""
        if a is None:
            return None, None
        if isinstance(a, torch.Tensor) and a.is_cuda:
            return a, None
        t = a if isinstance(a, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(a))
        if t.dtype == torch.bool:
            t = t.to(torch.uint8)
        pinned = t.pin_memory() if not t.is_pinned() else t
        with torch.cuda.stream(self.stream):
            d = torch.empty(t.shape, dtype=t.dtype, device="cuda")
            d.copy_(pinned, non_blocking=True)
            ev = torch.cuda.Event()
            ev.record(self.stream)
        with self.lock:
            self.h2d_bytes += t.numel() * t.element_size()
        return d, (ev, pinned)

    def prefetch(self, i: int):
        if i in self.pending:
            return
        dev = torch.cuda.current_device()

        def job():
            torch.cuda.set_device(dev)
            vol = self._stage(self.volumes[i])
            msk = self._stage(None if self.masks is None else self.masks[i])
            return vol, msk

        self.pending[i] = self.pool.submit(job)

    def get(self, i: int):
        """(volume, mask or None) of frame i on the device, ready for the current stream."""
        self.prefetch(i)
        vol, msk = self.pending[i].result()
        cur = torch.cuda.current_stream()
        out = []
        for d, ev in (vol, msk):
            if ev is not None:
                cur.wait_event(ev[0])
                d.record_stream(cur)
            out.append(d)
        return out[0], out[1]

    def drop(self, keep):
        """Forget the frames not in ``keep`` (their device copies are freed once the streams are done with them)."""
        for i in [k for k in self.pending if k not in keep]:
            self.pending.pop(i)

    def close(self):
        self.pool.shutdown(wait=True)
        self.pending.clear()


def _host(t):
    return None if t is None else t.detach().cpu().numpy()


def _fill_nan_rows(U: torch.Tensor, grid_shape) -> torch.Tensor:
    """utils/grid_interp.py:33-34: NaN nodes inpainted (spring model) before the grid is sampled."""
    bad = ~torch.isfinite(U).all(dim=1)
    if not bool(bad.any().item()):
        return U
    v = U.clone()
    v[bad] = 0.0
    _, err = K.inpaint(v, grid_shape, bad.to(torch.uint8).contiguous())
    errs = K.ErrorWords()
    errs.add(err, "inpaint")
    errs.check()
    return v


def compose_cumulative(frames: list, schedule: FrameSchedule, coords0: np.ndarray, axes: tuple, grid_shape, order: int = 3) -> None:
    """core/pipeline.py:455-491: fill ``U_accum`` of every frame by walking its reference chain to frame 0.  Frame k's
    displacement grid is interpolated (``order`` 3: cubic spline; 1: trilinear) at the positions its parent's
    material points have reached; frames against frame 0 keep their own U."""
    x0, y0, z0 = (np.asarray(a, dtype=np.float64) for a in axes)
    h = [float(a[1] - a[0]) if len(a) > 1 else 1.0 for a in (x0, y0, z0)]
    positions = {0: np.asarray(coords0, dtype=np.float64).copy()}
    for i, fr in enumerate(frames):
        frame = i + 1
        parent = schedule.parent(frame)
        pos_parent = positions.get(parent)
        if parent == 0 or pos_parent is None:
            fr.U_accum = fr.U.copy()
            positions[frame] = positions[0] + fr.U_accum
            continue
        U = _fill_nan_rows(torch.from_numpy(np.ascontiguousarray(fr.U)).cuda(), grid_shape)
        disp = K.grid_interp(U, grid_shape, (x0[0], y0[0], z0[0]), h, torch.from_numpy(pos_parent).cuda(), order)
        pos = pos_parent + disp.cpu().numpy()
        positions[frame] = pos
        fr.U_accum = pos - positions[0]


def frame_strains(frames: list, grid_shape, spacing, valid0: np.ndarray, elem_active0, sp: StrainParams, gauss_order: int = 2) -> None:
    """core/pipeline.py:421-433: the strain of every frame from its accumulated displacement on the node grid of the
    first frame's reference (its node validity; the frame's own F when its reference is frame 0), on the device."""
    from . import strain as ST
    from .mesh import surface_nodes

    boundary = np.zeros(int(np.prod(grid_shape)), dtype=bool)
    boundary[surface_nodes(grid_shape)] = True
    for fr in frames:
        F_direct = fr.F if fr.ref_frame == 0 else None
        out = ST.compute_strain_device(fr.U_accum, grid_shape, spacing, sp.method, tuple(sp.halfwidth), sp.strain_type,
                                       tuple(sp.voxel_size), torch.from_numpy(np.asarray(valid0, dtype=bool)), F_direct,
                                       torch.from_numpy(boundary), elem_active0, float(sp.disp_smoothing), float(sp.strain_smoothing),
                                       bool(sp.edge_trim), gauss_order)
        fr.strain = ST._result(_host(out["U_phys"]), _host(out["F_phys"]), _host(out["keep"]), sp.strain_type, out["method"], out)


def run_series(volumes, p: PL.PassParams, masks=None, schedule: FrameSchedule | None = None, reference_mode: str = "accumulative",
               cumulative_interp: str = "cubic", normalize: bool = True, strain: StrainParams | None = None) -> SeriesResult:
    """run_aldvc's sections 2-7 over ``volumes`` (frame 0 first; (nz, ny, nx) uint16 or float32 host arrays or CUDA
    tensors).  ``masks``: per frame, None or a material mask, used as the reference mask when the frame is a
    reference and as the deformed-frame mask when it is solved; ``schedule`` defaults to ``reference_mode``'s.
    ``strain``: StrainParams to add each frame's strain (of its accumulated displacement).  With ``p.tile_local`` > 0
    every pass is the tiled pass (tiling.run_pass_tiled) on host frames, for volumes beyond the device's memory.
    Returns a SeriesResult with one FrameResult per deformed frame."""
    n_frames = len(volumes)
    if n_frames < 2:
        raise ValueError(f"At least 2 volumes are required (got {n_frames}).")
    if schedule is None:
        schedule = FrameSchedule.from_mode(reference_mode, n_frames)
    elif len(schedule.ref_indices) != n_frames - 1:
        raise ValueError(f"frame_schedule length {len(schedule.ref_indices)} != n_frames-1 = {n_frames - 1}")
    if cumulative_interp not in ("linear", "cubic"):
        raise ValueError("cumulative_interp must be 'linear' or 'cubic'")
    shape = tuple(int(s) for s in volumes[0].shape)
    tiled = int(getattr(p, "tile_local", 0) or 0) > 0
    if tiled and any(isinstance(v, torch.Tensor) and v.is_cuda for v in volumes):
        raise ValueError("tile_local > 0: the frames of a tiled series stay in host memory")
    t_start = time.perf_counter()
    up = _Uploader(volumes, masks)
    refs: OrderedDict = OrderedDict()
    beta_by_ref: dict = {}
    frames: list = []
    prev_ref, prev_U = None, None
    timings: dict = {}
    valid0 = elem0 = spacing = None  # node validity and active elements of the first frame's reference, grid spacing
    try:
        if not tiled:
            up.prefetch(schedule.parent(1))
            up.prefetch(1)
        for k in range(1, n_frames):
            t_frame = time.perf_counter()
            ref_idx = schedule.parent(k)
            if k + 1 < n_frames and not tiled:  # the next frame (and a new reference) copy while this one is solved
                up.prefetch(k + 1)
                if schedule.parent(k + 1) not in refs:
                    up.prefetch(schedule.parent(k + 1))
            pk = p
            if p.beta is None and ref_idx in beta_by_ref:
                pk = copy.copy(p)
                pk.beta = beta_by_ref[ref_idx]
            previous = prev_U if prev_ref == ref_idx else None
            if tiled:  # volumes beyond the device: the frames stay in host memory, every pass streams its boxes
                from .tiling import run_pass_tiled

                res = run_pass_tiled(volumes[ref_idx], volumes[k], pk, None if masks is None else masks[ref_idx],
                                     None if masks is None else masks[k], normalize, previous=previous)
                ref_q = (res.H, res.valid, res.n_valid, res.bottomf, res.mesh, res.elem_active)
            else:
                if ref_idx in refs:
                    refs.move_to_end(ref_idx)
                else:
                    while len(refs) >= REF_CACHE:  # room first: a prepared reference holds about 17 bytes per voxel
                        refs.popitem(last=False)
                    f_d, m_d = up.get(ref_idx)
                    if tuple(f_d.shape) != shape:
                        raise ValueError(f"frame {ref_idx} has shape {tuple(f_d.shape)}, frame 0 {shape}")
                    t0 = time.perf_counter()
                    refs[ref_idx] = PL.prepare_reference(f_d, p, m_d, normalize)
                    timings["reference_prepare"] = timings.get("reference_prepare", 0.0) + time.perf_counter() - t0
                g_d, gm_d = up.get(k)
                if tuple(g_d.shape) != shape:
                    raise ValueError(f"frame {k} has shape {tuple(g_d.shape)}, frame 0 {shape}")
                rf = refs[ref_idx]
                res = PL.run_pass(None, g_d, pk, None, normalize, g_mask=gm_d, ref=rf, previous=previous)
                ref_q = (rf.H, rf.valid_b, rf.n_valid, rf.bottomf, rf.mesh, rf.elem_active)
            if p.beta is None and getattr(res, "beta", None) is not None:
                beta_by_ref.setdefault(ref_idx, float(res.beta))
            H_r, valid_r, n_valid_r, bottomf_r, mesh_r, elem_r = ref_q
            if valid0 is None:
                valid0, elem0, spacing = _host(valid_r), elem_r, mesh_r.spacing
            U_std = UN.displacement_uncertainty_device(H_r, res.zncc, res.status, valid_r, n_valid_r, bottomf_r, mesh_r.half,
                                                       p.subset_stride)
            frames.append(FrameResult(U=_host(res.U), F=_host(res.F), ref_frame=ref_idx, U_local=_host(res.U_local),
                                      F_local=_host(res.F_local), U0=_host(res.U0), zncc=_host(res.zncc), status=_host(res.status),
                                      outlier=_host(res.outlier), valid=_host(res.valid), beta=getattr(res, "beta", None),
                                      admm_steps=res.admm_steps, init_method=res.init_info.get("method", ""), U_std=_host(U_std)))
            prev_ref, prev_U = ref_idx, res.U
            # raw frames still to come: the next one and its reference when that is not prepared yet
            keep = {k + 1} | ({schedule.parent(k + 1)} if k + 1 < n_frames and schedule.parent(k + 1) not in refs else set())
            up.drop(keep)
            frames[-1].seconds = time.perf_counter() - t_frame
            timings[f"frame_{k}"] = frames[-1].seconds
    finally:
        up.close()
    x0, y0, z0 = build_grid_axes(shape, p.winsize, p.winstepsize)
    coords0 = grid_coords(x0, y0, z0)
    grid_shape = (len(z0), len(y0), len(x0))
    t7 = time.perf_counter()
    compose_cumulative(frames, schedule, coords0, (x0, y0, z0), grid_shape, 3 if cumulative_interp == "cubic" else 1)
    timings["cumulative"] = time.perf_counter() - t7
    if strain is not None:
        t8 = time.perf_counter()
        frame_strains(frames, grid_shape, spacing, valid0, elem0, strain, p.gauss_pt_order)
        timings["strain"] = time.perf_counter() - t8
    timings["h2d_bytes"] = up.h2d_bytes
    timings["total"] = time.perf_counter() - t_start
    return SeriesResult(frames, coords0, grid_shape, (x0, y0, z0), schedule, timings)
