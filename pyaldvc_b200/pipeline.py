"""One full AL-DVC pass on the device (pyALDVC core/pipeline.py:255-366, sections 3-6).

Every step runs in the library on CUDA tensors; the host only sequences the calls and, where the
reference makes a data-dependent decision (NCC radius expansion, the ADMM early stop), reads a few
scalars.  With ``admm_early_stop=False`` the ADMM loop makes no host decision at all and is
captured once as a CUDA graph (``graph=True``).

Parameter names and defaults follow ``DVCPara`` (core/config.py:36-162).
"""

from __future__ import annotations

import time
from dataclasses import dataclass

import numpy as np
import torch

from . import autotune
from . import beta_tuning as BT
from . import integer_search as IS
from . import kernels as K
from .mesh import build_grid_axes, grid_coords, surface_nodes

STATUS_CONVERGED = 0


@dataclass
class PassParams:
    winsize: tuple = (32, 32, 32)
    winstepsize: tuple = (16, 16, 16)
    search_radius: tuple = (8, 8, 8)
    init_subset: tuple | None = None  # None: min(winsize, 16) (init_disp.py:76-81)
    interp_method: str = "cubic"
    subset_stride: int = 1
    icgn_tol: float = 1e-2
    icgn_dp_tol: float = 1e-3
    icgn_max_iter: int = 100
    icgn_patience: int = 5
    icgn_predictive_stop: bool = True
    min_valid_ratio: float = 0.5
    hessian_cond_max: float = 1e12
    init_outlier_threshold: float = 2.0
    local_outlier_threshold: float = 2.0
    ncc_auto_expand: bool = True
    ncc_max_expand: int = 3
    use_global_step: bool = True
    mu: float = 1e-3
    beta: float | None = 1e-3  # None: tuned per pass over beta_range (solver/beta_tuning.py)
    beta_range: tuple = BT.DEFAULT_BETA_RANGE
    beta_criterion: str = "matlab"
    alpha: float = 0.0
    admm_max_iter: int = 4
    admm_tol: float = 1e-2
    admm_early_stop: bool = True
    dual_update: str = "accumulate"
    pcg_tol: float = 1e-8
    pcg_max_iter: int = 500
    gauss_pt_order: int = 2
    variant: int = K.BATCHED
    threads: int = 0  # 0: chosen by the autotuner (or the library default when autotune is off)
    brick_floats: int = 0
    autotune: bool = True
    icgn_sweep_rows: int = 0  # persistent IC-GN: subset rows per sweep tile (0 library default, < 0 C order)
    icgn_node_order: str = "morton"  # persistent IC-GN work queue: "morton" (nodes near each other solved together) or "index"
    icgn_quads: bool = True  # cubic / B-spline persistent IC-GN: sample g through its overlapping-quad copy
    graph: bool = False
    ncc_engine: str = "auto"  # auto | tiled | fft | fft_cluster | plain
    # uneven subsets: coords (N,3) [x, y, z] -> (N,3) even window sizes per node, each <= winsize (which then
    # sets the mesh border and the maximum shape); every shape runs in the same persistent launches
    node_winsize: object = None
    prefilter_sigma: float = 0.0  # Gaussian pre-smoothing of both volumes after normalisation (0 = off)
    # tiled pass (tiling.run_pass_tiled, core/config.py:140-142): box edge target in voxels (0 = one whole-volume
    # box), extra halo for the displacement (0 = max(winstepsize)), halo for the subset's stretch (fraction of
    # winsize / 2)
    tile_local: int = 0
    tile_disp_margin: int = 0
    tile_strain_margin: float = 0.25
    # initial guess (core/config.py:61-71): "pyramid" (coarse-to-fine NCC), "ncc" (one full-resolution search)
    # or "zero"; an optional global phase-correlation pre-shift
    init_guess_method: str = "pyramid"
    global_shift: bool = True
    pyramid_levels: int = 0  # 0: automatic
    pyramid_fine_radius: int = 2
    init_min_pce: float = 0.0


@dataclass
class PassResult:
    U: torch.Tensor
    F: torch.Tensor
    status: torch.Tensor
    zncc: torch.Tensor
    n_iter: torch.Tensor
    coords: torch.Tensor
    grid_shape: tuple
    valid: torch.Tensor
    U_local: torch.Tensor | None = None
    U0: torch.Tensor | None = None
    admm_steps: int = 0
    P_local: torch.Tensor | None = None  # raw 12-DOF result (before outlier filling)
    status_local: torch.Tensor | None = None
    n_iter_local: torch.Tensor | None = None


class Tracer:
    """Stage timing: CUDA events on the current stream (no synchronisation) or, with ``sync=True``,
    wall clock after a device synchronisation.  ``stages()`` returns seconds per stage."""

    def __init__(self, sync: bool = False):
        self.sync = sync
        self.marks: list = []
        self._t0 = None

    def start(self):
        if self.sync:
            torch.cuda.synchronize()
            self._t0 = time.perf_counter()
        else:
            e = torch.cuda.Event(enable_timing=True)
            e.record()
            self._t0 = e

    def mark(self, name: str):
        if self.sync:
            torch.cuda.synchronize()
            t = time.perf_counter()
            self.marks.append((name, t - self._t0))
            self._t0 = t
        else:
            e = torch.cuda.Event(enable_timing=True)
            e.record()
            self.marks.append((name, self._t0, e))
            self._t0 = e

    def stages(self) -> dict:
        out: dict = {}
        for m in self.marks:
            dt = m[1] if self.sync else m[1].elapsed_time(m[2]) / 1e3
            out[m[0]] = out.get(m[0], 0.0) + dt
        return out


class Mesh:
    """Node grid + reference-derived per-node data (the ``LocalContext`` of local_icgn.py:40-93)."""

    def __init__(self, volume_shape, p: PassParams, voi=None):
        x0, y0, z0 = build_grid_axes(volume_shape, p.winsize, p.winstepsize, voi)
        self.grid_shape = (len(z0), len(y0), len(x0))
        self.spacing = (float(x0[1] - x0[0]), float(y0[1] - y0[0]), float(z0[1] - z0[0]))
        self.coords_np = np.round(grid_coords(x0, y0, z0)).astype(np.int64)
        self.axes = tuple(np.round(np.asarray(a, dtype=np.float64)).astype(np.int64) for a in (x0, y0, z0))  # xs, ys, zs
        self.coords = torch.from_numpy(self.coords_np).cuda()
        self.axes_dev = tuple(torch.from_numpy(a).cuda() for a in self.axes)
        self.n = self.coords_np.shape[0]
        self.half = tuple(int(w) // 2 for w in p.winsize)
        self._order = None

    def order(self) -> torch.Tensor:
        """(N,) int32 CUDA tensor: the nodes sorted by the Morton code of their grid position (z, y, x bits
        interleaved), so that nodes handed out together by a work queue lie in compact blocks of the volume."""
        if self._order is None:
            key = (self.grid_shape, torch.cuda.current_device())
            if key not in _MORTON:
                nz, ny, nx = self.grid_shape
                iz, iy, ix = (a.ravel().astype(np.uint64) for a in np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx),
                                                                                indexing="ij"))
                code = np.zeros(self.n, dtype=np.uint64)
                for b in range(21):
                    for k, v in enumerate((ix, iy, iz)):
                        code |= ((v >> np.uint64(b)) & np.uint64(1)) << np.uint64(3 * b + k)
                while len(_MORTON) >= 4:
                    _MORTON.pop(next(iter(_MORTON)))
                _MORTON[key] = torch.from_numpy(np.argsort(code, kind="stable").astype(np.int32)).cuda()
            self._order = _MORTON[key]
        return self._order


_MORTON: dict = {}  # Morton node orders by (grid shape, device), the few most recent


def _fill(values: torch.Tensor, bad: torch.Tensor, grid_shape, errs: K.ErrorWords):
    """fill_bad_nodes / clean_initial_guess inpainting of the rows flagged in ``bad`` (all bad -> zeros)."""
    unk = bad.to(torch.uint8).contiguous()
    v = values.clone().contiguous()
    v[bad] = 0.0
    _, e = K.inpaint(v, grid_shape, unk)
    errs.add(e, "inpaint")
    return v, bad.all()


def _median_flags(field: torch.Tensor, good: torch.Tensor, grid_shape, threshold, errs: K.ErrorWords):
    if threshold <= 0:
        return torch.zeros_like(good)
    f, e = K.median_test(field.contiguous(), grid_shape, good.to(torch.uint8).contiguous(), threshold)
    errs.add(e, "median_test")
    # the reference runs the test only with more than 27 good nodes (local_icgn.py:469-475)
    return (f != 0) & (good.sum() > 27)


def _rms(a: torch.Tensor) -> torch.Tensor:
    return torch.sqrt(torch.mean(a * a))


# integer_search.py:395: the reference's CPU search switches from the direct map to FFTs above this many
# template-voxel x offset products per node
FFT_NCC_MIN_OPS = 3e7


def _ncc_engine(p: PassParams, half, radius) -> int:
    """NCC engine of a search: the plain form's map kernel, or by ``p.ncc_engine``; ``auto`` takes the FFT
    engine for searches of more than ``FFT_NCC_MIN_OPS`` multiply-adds per node, else the tiled direct engine."""
    if p.variant == K.PLAIN or p.ncc_engine == "plain":
        return K.NCC_PLAIN
    if p.ncc_engine in ("tiled", "fft", "fft_cluster"):
        return {"tiled": K.NCC_TILED, "fft": K.NCC_FFT, "fft_cluster": K.NCC_FFT_CLUSTER}[p.ncc_engine]
    n_tpl = np.prod([2 * int(h) + 1 for h in half])
    n_off = np.prod([2 * int(r) + 1 for r in radius])
    return K.NCC_FFT if n_tpl * n_off > FFT_NCC_MIN_OPS else K.NCC_TILED


def _launch_shape(p: PassParams, ndof: int, mode: int, mesh, mask, run) -> tuple[int, int]:
    """(threads, brick_floats) of the batched IC-GN launches: the caller's, else the autotuner's choice for
    this kernel and subset, timed on an evenly spread sample of this pass's nodes."""
    if p.variant != K.BATCHED or p.threads != 0 or not p.autotune or p.node_winsize is not None:
        return p.threads, p.brick_floats  # per-node shapes always run the lean kernel
    k = autotune.key(ndof, mode, True, mesh.half, p.subset_stride, mask is not None, mesh.n)
    idx = autotune.sample_index(mesh.n)
    return autotune.tune(k, lambda th, br: run(idx, th, br))


# captured ADMM loops, keyed by problem shape and parameters (the oldest is dropped beyond the limit)
ADMM_GRAPH_CACHE = 2
_ADMM_GRAPHS: dict = {}


def _graph_key(p: PassParams, mesh, mode, th3, br3, n_full, tensors, beta) -> tuple:
    shapes = tuple((k, None if t is None else (tuple(t.shape), str(t.dtype))) for k, t in sorted(tensors.items()))
    prm = (beta, p.mu, p.alpha, p.pcg_tol, p.pcg_max_iter, p.gauss_pt_order, p.icgn_tol, p.icgn_dp_tol, p.icgn_max_iter,
           p.icgn_patience, p.icgn_predictive_stop, p.admm_max_iter, p.dual_update, p.local_outlier_threshold, p.subset_stride,
           p.variant, p.icgn_sweep_rows, p.icgn_node_order, p.icgn_quads)
    return (mesh.grid_shape, tuple(mesh.half), tuple(mesh.spacing), mode, th3, br3, n_full, prm, shapes)


def clear_graphs() -> None:
    """Release every captured ADMM loop (and the device memory its static tensors hold)."""
    _ADMM_GRAPHS.clear()


def graph_count() -> int:
    """Number of captured ADMM loops currently cached."""
    return len(_ADMM_GRAPHS)


def node_validity(mesh, p: PassParams, node_half, valid_b: torch.Tensor, centre_ok: torch.Tensor | None, n_valid: torch.Tensor):
    """(node validity, active elements uint8 or None): with a reference mask (``centre_ok`` set) apply_mask_to_mesh
    (grid_mesh.py:191-253) keeps the nodes whose centre is in the mask and enough of whose subset is, and the hex
    elements whose eight nodes are kept; without one every node and element stays."""
    if centre_ok is None:
        return valid_b, None
    if node_half is None:
        S = float(np.prod([2 * h + 1 for h in mesh.half]))
    else:
        S = (2 * node_half.double() + 1).prod(dim=1)
    node_valid = centre_ok & (n_valid.double() >= p.min_valid_ratio * S)
    valid_b = valid_b & node_valid
    elem_node = node_valid.reshape(mesh.grid_shape)
    e = (elem_node[:-1, :-1, :-1] & elem_node[:-1, :-1, 1:] & elem_node[:-1, 1:, 1:] & elem_node[:-1, 1:, :-1]
         & elem_node[1:, :-1, :-1] & elem_node[1:, :-1, 1:] & elem_node[1:, 1:, 1:] & elem_node[1:, 1:, :-1])
    return valid_b, e.reshape(-1).to(torch.uint8).contiguous()


def initial_guess(p: PassParams, mesh, f, g, search_valid: torch.Tensor, ncc_calls: list, errs: K.ErrorWords, shift_fn=None,
                  search_fn=None, level_volumes=None, levels: int | None = None, previous: torch.Tensor | None = None):
    """Section 3 of the pass (init_disp.compute_initial_guess :53-140, clean_initial_guess :143-189): (U0 (N,3)
    FP64, record).  ``f``, ``g``: the normalised device pair, or shape-only stand-ins when ``shift_fn`` (the global
    shift), ``search_fn`` (full-resolution searches), ``level_volumes`` (coarse pyramid pairs) and ``levels`` come
    from a pass that streams its volumes (tiling.run_pass_tiled)."""
    subset0 = p.init_subset if p.init_subset is not None else tuple(min(int(w), 16) for w in p.winsize)
    half0 = tuple(int(w) // 2 for w in subset0)
    rad = tuple(int(r) for r in p.search_radius)
    engine_of = lambda h, r: _ncc_engine(p, h, r)  # noqa: E731
    if p.init_guess_method not in ("pyramid", "ncc", "zero", "previous"):
        raise ValueError(f"unknown init_guess_method {p.init_guess_method!r}")
    if p.init_guess_method == "zero":
        return torch.zeros((mesh.n, 3), dtype=torch.float64, device="cuda"), {"method": "zero"}
    # the last frame's field when it was solved against the same reference and is finite everywhere, as it is (no
    # cleaning); otherwise the pyramid (init_disp.py:70-73)
    if p.init_guess_method == "previous" and previous is not None and tuple(previous.shape) == (mesh.n, 3) \
            and bool(torch.isfinite(previous).all().item()):
        return previous.to(device="cuda", dtype=torch.float64).clone(), {"method": "previous"}
    shift = None
    if p.global_shift:
        shift = shift_fn() if shift_fn is not None else IS.phase_correlation_shift_device(f, g)
    if p.init_guess_method in ("pyramid", "previous"):  # "previous" without a usable field: the pyramid
        info = IS.pyramid_search_device(f, g, mesh.coords, mesh.grid_shape, subset0, rad,
                                        p.pyramid_levels if levels is None else levels, shift, p.init_outlier_threshold,
                                        p.ncc_auto_expand, p.ncc_max_expand, p.pyramid_fine_radius, search_valid, engine_of, ncc_calls,
                                        errs, level_volumes, search_fn)
        disp, ok, pce = info["disp"], info.get("ok"), info.get("pce")
        if ok is None:
            ok = torch.ones(mesh.n, dtype=torch.bool, device="cuda")
        init_info = {"method": "pyramid", "levels": info["levels"], "per_level": info["per_level"], "expansions": info["expansions"]}
    else:
        act = torch.nonzero(search_valid).flatten()
        if act.numel() == 0:
            act = torch.arange(mesh.n, device="cuda")
        sh0 = None
        if shift is not None:
            sh0 = torch.as_tensor(np.round(shift).astype(np.int64), device="cuda")[None, :].expand(act.numel(), 3).contiguous()
        res = IS.ncc_search_expanding_device(f, g, mesh.coords[act].contiguous(), half0, rad, sh0, p.ncc_auto_expand,
                                             p.ncc_max_expand, engine_of, ncc_calls, search_fn)
        disp = torch.full((mesh.n, 3), float("nan"), dtype=torch.float64, device="cuda")
        ok = torch.zeros(mesh.n, dtype=torch.bool, device="cuda")
        pce = torch.full((mesh.n,), float("nan"), dtype=torch.float64, device="cuda")
        disp[act] = res["disp"]
        ok[act] = res["ok"]
        pce[act] = res["pce"]
        init_info = {"method": "ncc", "radius": res["radius"], "expansions": res["expansions"]}
    init_info["global_shift"] = shift
    bad = ~ok | ~torch.isfinite(disp).all(dim=1) | ~search_valid
    if p.init_min_pce > 0 and pce is not None:
        bad = bad | (torch.isfinite(pce) & (pce < p.init_min_pce))
    flag = _median_flags(torch.where(bad[:, None], torch.nan, disp), ~bad, mesh.grid_shape, p.init_outlier_threshold, errs)
    bad = bad | flag
    U0, all_bad = _fill(disp, bad, mesh.grid_shape, errs)
    if bool(all_bad.item()):
        U0.zero_()
    init_info["n_bad"] = int(bad.sum().item())
    return U0, init_info


def make_global_step(mesh, p: PassParams, elem_active, beta, errs: K.ErrorWords):
    """The global step of one ADMM iteration (subpb2_solver.py, pipeline.py:300-330): right-hand side, hex8 PCG from
    U1, nodal gradient of the result (non-finite entries keep F1).  Returns a function (U1, F1, W, v) -> (U2, F2)."""

    def global_step(U1_, F1_, W_, v_):
        b = K.global_rhs(mesh.grid_shape, mesh.spacing, elem_active, beta, p.mu, p.alpha, U1_, F1_, W_, v_, p.gauss_pt_order)
        U2_, _, e_ = K.pcg_hex8(mesh.grid_shape, mesh.spacing, elem_active, beta, p.mu, p.alpha, b, U1_, p.pcg_tol, p.pcg_max_iter,
                                p.gauss_pt_order)
        errs.add(e_, "pcg_hex8")
        F2_ = K.nodal_gradient(mesh.grid_shape, mesh.spacing, elem_active, U2_, p.gauss_pt_order).reshape(-1, 9)
        F2_ = torch.where(torch.isfinite(F2_), F2_, F1_)
        return U2_, F2_

    return global_step


@dataclass
class Reference:
    """A reference frame prepared for any number of deformed frames (core/pipeline.py:187-228 get_reference): the
    normalised (and presmoothed) volume, its gradients and mask, the node grid, the per-node precompute and the node
    and element validity.  ``key`` holds the parameters it was prepared with."""

    f: torch.Tensor
    gx: torch.Tensor
    gy: torch.Tensor
    gz: torch.Tensor
    m_u8: torch.Tensor | None
    mesh: Mesh
    node_half: torch.Tensor | None
    H: torch.Tensor
    L: torch.Tensor
    meanf: torch.Tensor
    bottomf: torch.Tensor
    n_valid: torch.Tensor
    valid_b: torch.Tensor
    elem_active: torch.Tensor | None
    precompute_form: str
    key: tuple


_COPY_STREAMS: dict = {}


def _upload_inputs(*inputs):
    """Device copies of the host (CPU) tensors among a pass's inputs, issued in argument order on a copy stream of
    this device; CUDA tensors and None pass through.  Each block is allocated on the current stream and recorded on
    the copy stream, and the copy stream first waits for the current stream's queued work (a block may come from a
    tensor that work still reads).  Returns the tensors and, per argument, the event after its copy (None where
    nothing was copied).  From pinned host memory the copies run behind the kernels queued meanwhile; from pageable
    memory each copy returns only once it is done.  Host-to-device copies share a copy engine in issue order: a
    small copy issued after these (node coordinates and the like) waits for all of them, so the caller makes its
    own small copies first."""
    dev = torch.cuda.current_device()
    cs = _COPY_STREAMS.get(dev)
    if cs is None:
        cs = _COPY_STREAMS[dev] = torch.cuda.Stream()
    cs.wait_stream(torch.cuda.current_stream())
    out, evs = [], []
    for t in inputs:
        if t is None or t.is_cuda:
            out.append(t)
            evs.append(None)
            continue
        d = torch.empty(t.shape, dtype=t.dtype, device="cuda")
        d.record_stream(cs)
        with torch.cuda.stream(cs):
            d.copy_(t, non_blocking=True)
            ev = torch.cuda.Event()
            ev.record(cs)
        out.append(d)
        evs.append(ev)
    return out, evs


def _reference_key(p: PassParams, normalize: bool, shape) -> tuple:
    return (tuple(int(s) for s in shape), tuple(p.winsize), tuple(p.winstepsize), p.min_valid_ratio, p.hessian_cond_max,
            p.subset_stride, p.variant, id(p.node_winsize) if p.node_winsize is not None else None, p.prefilter_sigma, bool(normalize))


def prepare_reference(f_raw: torch.Tensor, p: PassParams, mask: torch.Tensor | None = None, normalize: bool = True,
                      tracer: Tracer | None = None, mesh: Mesh | None = None) -> Reference:
    """Normalisation, presmoothing, gradients, node grid, precompute (local_icgn.precompute_local_context :223-347)
    and node validity (grid_mesh.apply_mask_to_mesh) of a reference frame on the device.  ``tracer`` is marked
    "preprocess" after the volume work and "precompute" at the end.  ``mesh``: the node grid of this volume shape
    and these parameters, when the caller made it already."""
    f = K.normalize(f_raw) if normalize else f_raw.float().contiguous()
    if p.prefilter_sigma and p.prefilter_sigma > 0:  # core/pipeline.py:197
        f = K.gaussian_presmooth(f, p.prefilter_sigma)
    gx, gy, gz = K.gradients(f)
    if mesh is None:
        mesh = Mesh(f.shape, p)
    m_u8 = None if mask is None else mask.to(torch.uint8).contiguous()
    if tracer is not None:
        tracer.mark("preprocess")
    node_half = None
    if p.node_winsize is not None:
        ws = np.asarray(p.node_winsize(mesh.coords.cpu().numpy()), dtype=np.int64).reshape(-1, 3)
        hs = ws // 2
        if (hs > np.asarray(mesh.half)[None, :]).any():
            raise ValueError("node_winsize exceeds winsize")
        node_half = torch.from_numpy(hs.astype(np.int32)).cuda()
    nz_, ny_, nx_ = f.shape
    if node_half is None and p.subset_stride == 1 and p.variant == K.BATCHED and nx_ <= 8192 and ny_ <= 65535:
        # a tensor grid of nodes with one subset shape: separable moment sums (the batched form)
        H, L, meanf, bottomf, n_valid, valid = K.precompute_grid(*mesh.axes_dev, mesh.half, f, gx, gy, gz, p.min_valid_ratio,
                                                                 p.hessian_cond_max, m_u8)
        precompute_form = "grid"
    else:
        precompute_form = "per_node"
        H, L, meanf, bottomf, n_valid, valid = K.precompute(mesh.coords, mesh.half, f, gx, gy, gz, m_u8, p.min_valid_ratio,
                                                            p.hessian_cond_max, p.subset_stride, None, None, node_half)
    centre_ok = None
    if mask is not None:
        c = mesh.coords
        centre_ok = m_u8[c[:, 2], c[:, 1], c[:, 0]] != 0
    valid_b, elem_active = node_validity(mesh, p, node_half, valid != 0, centre_ok, n_valid)
    if tracer is not None:
        tracer.mark("precompute")
    return Reference(f, gx, gy, gz, m_u8, mesh, node_half, H, L, meanf, bottomf, n_valid, valid_b, elem_active, precompute_form,
                     _reference_key(p, normalize, f_raw.shape))


def run_pass(f_raw: torch.Tensor | None, g_raw: torch.Tensor, p: PassParams, mask: torch.Tensor | None = None, normalize: bool = True,
             tracer: Tracer | None = None, g_mask: torch.Tensor | None = None, ref: Reference | None = None,
             previous: torch.Tensor | None = None) -> PassResult:
    """Full pass on one volume pair ((nz, ny, nx) float32 or uint16 tensors, on the device or in host memory).
    ``mask``: reference-frame material mask; ``g_mask``: deformed-frame mask (False voxels are excluded from every
    correlation).  ``ref``: the reference frame prepared by ``prepare_reference`` (then ``f_raw`` and ``mask`` are
    not read); ``previous``: the displacement field (N, 3) of the last frame solved against the same reference, the
    initial guess of ``init_guess_method="previous"`` (core/pipeline.py:266, init_disp.py:70-73).  Host inputs are
    copied within the pass, the reference frame first: its preparation runs while the deformed frame is copied
    (pinned host memory lets the two overlap)."""
    tr = tracer if tracer is not None else Tracer(sync=False)
    tr.start()
    # device error words of the bounded waits (inpainting, median test, PCG), read once at the end of the pass
    errs = K.ErrorWords()
    g_ready = None
    mesh0 = None
    if any(t is not None and not t.is_cuda for t in (f_raw, g_raw, mask, g_mask)):
        if ref is not None:
            f_raw = mask = None
        else:  # the node grid's own small copies go ahead of the volumes' in the copy engine's queue
            mesh0 = Mesh(tuple(f_raw.shape), p)
        (f_raw, mask, g_raw, g_mask), evs = _upload_inputs(f_raw, mask, g_raw, g_mask)
        cur = torch.cuda.current_stream()
        for ev in evs[:2]:
            if ev is not None:
                cur.wait_event(ev)
        g_ready = [ev for ev in evs[2:] if ev is not None]
    mode = K.INTERP_MODE_BY_NAME[p.interp_method]

    def prepare_deformed():
        g_ = K.normalize(g_raw) if normalize else g_raw.float().contiguous()
        if p.prefilter_sigma and p.prefilter_sigma > 0:  # core/pipeline.py:257
            g_ = K.gaussian_presmooth(g_, p.prefilter_sigma)
        # the array the interpolation samples, and the NCC input (core/pipeline.py:258-262, io/volume_ops.py:225-244)
        gp_ = K.bspline_prefilter(g_) if p.interp_method == "bspline" else g_
        if g_mask is not None:
            gm = g_mask.to(torch.uint8).contiguous()
            if gp_ is g_:
                gp_ = g_.clone()
            K.mask_fill(gp_, gm, float("nan"))
            g_ = K.mask_fill(g_.clone(), gm, 0.0)
        return g_, gp_

    if g_ready is None:
        g, g_prep = prepare_deformed()
    if ref is None:
        ref = prepare_reference(f_raw, p, mask, normalize, tr, mesh=mesh0)
    else:
        if ref.key != _reference_key(p, normalize, g_raw.shape):
            raise ValueError("run_pass: the prepared reference was made with other parameters or another volume shape")
        tr.mark("preprocess")
        tr.mark("precompute")
    if g_ready is not None:
        for ev in g_ready:
            torch.cuda.current_stream().wait_event(ev)
        g, g_prep = prepare_deformed()
        tr.mark("preprocess")
    f, gx, gy, gz, m_u8, mesh, node_half = ref.f, ref.gx, ref.gy, ref.gz, ref.m_u8, ref.mesh, ref.node_half
    H, L, meanf, bottomf, n_valid = ref.H, ref.L, ref.meanf, ref.bottomf, ref.n_valid
    valid_b, elem_active, precompute_form = ref.valid_b, ref.elem_active, ref.precompute_form
    valid_u8 = valid_b.to(torch.uint8).contiguous()

    # ---------------- section 3: initial guess (init_disp.compute_initial_guess :53-140, clean_initial_guess :143-189)
    # the reference makes the precompute's validity the mesh's node validity before the initial guess
    # (core/pipeline.py:212, local_icgn.py:300): only those nodes are searched, the others are filled
    ncc_calls: list = []
    U0, init_info = initial_guess(p, mesh, f, g, valid_b, ncc_calls, errs, previous=previous)
    tr.mark("init_guess")

    # ---------------- section 4: local 12-DOF IC-GN (local_icgn.local_icgn :398-489)
    # the persistent kernels read each cubic tap row of g as one 16-byte load from its overlapping-quad copy
    g4 = K.make_quads(g_prep) if (mode != 0 and p.variant == K.BATCHED and p.icgn_quads) else None
    order = mesh.order() if (p.variant == K.BATCHED and p.icgn_node_order == "morton") else None
    P0 = torch.zeros((mesh.n, 12), dtype=torch.float64, device="cuda")
    P0[:, 9:] = U0

    def icgn12_on(idx, th, br):
        c, P0_, L_, mf_, v_ = ((mesh.coords, P0, L, meanf, valid_u8) if idx is None else
                               (mesh.coords[idx], P0[idx], L[idx], meanf[idx], valid_u8[idx]))
        nh = node_half if (node_half is None or idx is None) else node_half[idx]
        return K.icgn12(c, P0_, mesh.half, f, gx, gy, gz, m_u8, g_prep, mode, L_, mf_, v_, p.icgn_tol, p.icgn_dp_tol, p.icgn_max_iter,
                        p.icgn_patience, p.subset_stride, None, None, 0.0, p.icgn_predictive_stop, None, None, p.variant, th, br,
                        node_half=nh, g4=g4, sweep_rows=p.icgn_sweep_rows, node_order=order if idx is None else None,
                        errs=errs if idx is None else None)

    th12, br12 = _launch_shape(p, 12, mode, mesh, m_u8, lambda idx, th, br: icgn12_on(idx, th, br))
    P, n_iter, status, zncc = icgn12_on(None, th12, br12)
    bad = status != STATUS_CONVERGED
    flag = _median_flags(P[:, 9:].contiguous(), ~bad, mesh.grid_shape, p.local_outlier_threshold, errs)
    bad = bad | flag
    UF, all_bad = _fill(P, bad, mesh.grid_shape, errs)  # U and F inpainted together (fill_bad_nodes :492-522)
    if bool(all_bad.item()):
        UF.zero_()
    U1 = UF[:, 9:].contiguous()
    F1 = UF[:, :9].contiguous()
    U_local = U1.clone()
    tr.mark("local_icgn")

    result = PassResult(U=U1, F=F1.reshape(-1, 3, 3), status=status, zncc=zncc, n_iter=n_iter, coords=mesh.coords,
                        grid_shape=mesh.grid_shape, valid=valid_b, U_local=U_local, U0=U0, P_local=P, status_local=status,
                        n_iter_local=n_iter)
    result.F_local = F1.reshape(-1, 3, 3).clone()  # the local result after outlier filling
    # converged, then rejected by the median test and replaced: not a measurement (core/pipeline.py:369-370)
    result.outlier = bad & (status == STATUS_CONVERGED)
    result.tracer = tr
    result.ncc_calls = ncc_calls  # (nodes, half, radius, engine) of every integer search of the pass
    result.init_info = init_info
    result.precompute_form = precompute_form
    result.node_half = node_half
    result.icgn3_iters = []  # n_iter tensors of every 3-DOF pass
    if not p.use_global_step:
        errs.check()
        return result

    # ---------------- sections 5-6: ADMM (pipeline.py:286-352), beta fixed or tuned (pipeline.py:288-298)
    beta = p.beta
    result.beta_sweep = None
    if beta is None:
        exclude = bad.clone()
        exclude[torch.from_numpy(surface_nodes(mesh.grid_shape)).cuda()] = True
        beta, result.beta_sweep = BT.auto_tune_beta_device(mesh.grid_shape, mesh.spacing, elem_active, p.mu, p.alpha, U1, F1, exclude,
                                                           p.winstepsize, p.beta_range, p.beta_criterion, p.pcg_tol, p.pcg_max_iter,
                                                           p.gauss_pt_order)
    result.beta = beta
    n_full = float(np.prod([(2 * h) // p.subset_stride + 1 for h in mesh.half]))
    # every tensor the ADMM loop reads; a captured loop reads static copies of them
    T = {"f": f, "g": g_prep, "gx": gx, "gy": gy, "gz": gz, "m": m_u8, "H": H, "meanf": meanf, "bottomf": bottomf, "valid": valid_u8,
         "coords": mesh.coords, "elem": elem_active, "node_half": node_half, "g4": g4, "order": order}

    def make_steps(T, errs_):
        global_step = make_global_step(mesh, p, T["elem"], beta, errs_)

        def icgn3_on(idx, U2_, F2_, v_, th, br):
            keys = ("coords", "H", "meanf", "bottomf", "valid")
            c, H_, mf_, bf_, ok_ = (T[k] if idx is None else T[k][idx] for k in keys)
            if idx is not None:
                U2_, F2_, v_ = U2_[idx], F2_[idx], v_[idx]
            nh = T["node_half"] if (T["node_half"] is None or idx is None) else T["node_half"][idx]
            return K.icgn3(c, U2_, F2_, v_, mesh.half, T["f"], T["gx"], T["gy"], T["gz"], T["m"], T["g"], mode, H_, mf_, bf_, ok_,
                           p.mu, p.icgn_tol, p.icgn_dp_tol, p.icgn_max_iter, p.icgn_patience, p.subset_stride, n_full, 0.0,
                           p.icgn_predictive_stop, None, None, p.variant, th, br, node_half=nh, g4=T["g4"],
                           sweep_rows=p.icgn_sweep_rows, node_order=T["order"] if idx is None else None,
                           errs=errs_ if idx is None else None)

        def admm_step(U2, F2, W, v, th3, br3):
            # subproblem 1 (subpb1_solver.subpb1_solver :77-164)
            U, it3, st3, zc3 = icgn3_on(None, U2, F2, v, th3, br3)
            bad3 = st3 != STATUS_CONVERGED
            bad3 = bad3 | _median_flags(U, ~bad3, mesh.grid_shape, p.local_outlier_threshold, errs_)
            U1n = torch.where(bad3[:, None], U2, U)
            F1n = F2
            U2n, F2n = global_step(U1n, F1n, W, v)
            if p.dual_update == "accumulate":
                Wn = W + (F2n - F1n)
                vn = v + (U2n - U1n)
            else:
                Wn = F2n - F1n
                vn = U2n - U1n
            du_g = _rms(U2n - U2)
            return U1n, U2n, F2n, Wn, vn, du_g, st3, zc3, it3, bad3

        return global_step, icgn3_on, admm_step

    global_step, icgn3_on, admm_step = make_steps(T, errs)
    W = torch.zeros((mesh.n, 9), dtype=torch.float64, device="cuda")
    v = torch.zeros((mesh.n, 3), dtype=torch.float64, device="cuda")
    U2, F2 = global_step(U1, F1, W, v)
    W = F2 - F1
    v = U2 - U1
    th3, br3 = _launch_shape(p, 3, mode, mesh, m_u8, lambda idx, th, br: icgn3_on(idx, U2, F2, v, th, br))

    steps = 1
    st_last, zc_last, it_last, bad_last = status, zncc, n_iter, bad
    U1_prev = U1
    if p.graph and not p.admm_early_stop and p.admm_max_iter > 1:
        # the remaining loop as one CUDA graph, captured on the first pass of this problem shape and replayed
        # by every later one after its inputs are copied into the graph's static tensors (no host step inside)
        state = {"U2": U2, "F2": F2, "W": W, "v": v}
        key = _graph_key(p, mesh, mode, th3, br3, n_full, {**T, **state}, beta)
        entry = _ADMM_GRAPHS.get(key)
        if entry is None:
            static = {k: (None if t is None else t.clone()) for k, t in {**T, **state}.items()}
            warm_errs, graph_errs = K.ErrorWords(), K.ErrorWords()
            _, _, admm_static = make_steps(static, warm_errs)
            side = torch.cuda.Stream()
            side.wait_stream(torch.cuda.current_stream())
            with torch.cuda.stream(side):  # warm-up outside capture (allocator pools, kernel attributes)
                admm_static(static["U2"], static["F2"], static["W"], static["v"], th3, br3)
            torch.cuda.current_stream().wait_stream(side)
            warm_errs.check()
            _, _, admm_static = make_steps(static, graph_errs)
            graph = torch.cuda.CUDAGraph()
            with torch.cuda.graph(graph):
                a = (static["U2"], static["F2"], static["W"], static["v"])
                outs = []
                for _ in range(2, p.admm_max_iter + 1):
                    U1g, U2g, F2g, Wg, vg, _, stg, zcg, itg, bdg = admm_static(*a, th3, br3)
                    outs.append((U1g, stg, zcg, itg, bdg))
                    a = (U2g, F2g, Wg, vg)
            entry = {"graph": graph, "static": static, "final": a, "outs": outs[-1], "iters": [o[3] for o in outs],
                     "errs": graph_errs}
            _ADMM_GRAPHS[key] = entry
            while len(_ADMM_GRAPHS) > ADMM_GRAPH_CACHE:
                _ADMM_GRAPHS.pop(next(iter(_ADMM_GRAPHS)))
            tr.mark("admm_capture")
        else:
            for k, t in {**T, **state}.items():
                if t is not None:
                    entry["static"][k].copy_(t)
        entry["graph"].replay()
        errs.extend(entry["errs"])  # the graph's error words, rewritten by this replay
        # the graph's outputs are overwritten by its next replay: the result keeps copies
        U2, F2 = entry["final"][0].clone(), entry["final"][1].clone()
        U1, st_last, zc_last, it_last, bad_last = (t.clone() for t in entry["outs"])
        result.icgn3_iters = [t.clone() for t in entry["iters"]]
        steps = p.admm_max_iter
    else:
        for step in range(2, p.admm_max_iter + 1):
            steps = step
            U1n, U2n, F2n, W, v, du_g, st_last, zc_last, it_last, bad_last = admm_step(U2, F2, W, v, th3, br3)
            result.icgn3_iters.append(it_last)
            du_l = _rms(U1n - U1_prev)
            U1_prev = U1n
            U1, U2, F2 = U1n, U2n, F2n
            if p.admm_early_stop and (float(du_g.item()) < p.admm_tol or float(du_l.item()) < p.admm_tol):
                break
    errs.check()
    tr.mark("admm")
    result.U = U2
    result.F = F2.reshape(-1, 3, 3)
    result.status, result.zncc, result.n_iter = st_last, zc_last, it_last
    result.admm_steps = steps
    result.outlier = bad_last & (st_last == STATUS_CONVERGED)
    return result
