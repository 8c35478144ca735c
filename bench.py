"""Benchmark: nodes/s of a full AL-DVC pass on one B200 (batched form), beside the plain form and the CPU oracle.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--config 5] [--impl reference]

A step is one full pass (normalise, gradients, NCC initial guess with cleaning, precompute, 12-DOF local
IC-GN with outlier filling, ADMM: global hex8 PCG + 3-DOF subproblem 1) over the configuration's volume
pair, inputs resident in HBM.  Rank 0 prints one JSON line.  With N > 1 (torchrun) every rank runs its own
replica of the workload (weak scaling; the pass needs no exchange between replicas); the value is the
nodes of all ranks over the slowest rank's time.
"""

from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

METRIC = "nodes/s full AL-DVC pass at <=0.01 vox RMS err; batched vs plain form, 1 B200"
WORKLOAD = {
    1: "64^3 bead pair, translation, ws20/st8, trilinear, NCC +-4, local IC-GN (125 nodes)",
    2: "128^3 bead pair, 2% z strain + sine, ws24/st6, tricubic, NCC +-8, local IC-GN (4096 nodes)",
    3: "256^3 uint16 bead pair, 5 deg rotation + 1% hydrostatic, sphere ROI r110, uneven subsets 16x16x24..32^3/st8, 3 ADMM (graph)",
    4: "192^3 bead pair, 10000 random 21^3 subsets, random affine warps, ZNSSD forward + backward (P and g), tricubic",
    5: "1024x1024x306 uint16 confocal-like bead pair, Boussinesq indentation, ws32/st12, NCC +-16, tricubic, 3 ADMM",
}
ZNSSD_METRIC = "subsets/s ZNSSD forward+backward (torch.autograd.Function), 1 B200"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--config", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--plain-steps", type=int, default=1, help="timed passes of the plain form (0 skips it)")
    ap.add_argument("--cpu-nodes", type=int, default=8, help="node block edge of the CPU baseline sample (cube root)")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--icgn-threads", type=int, default=0,
                    help="pin the batched IC-GN kernels to the lean form with this many threads per node (32/64/128) "
                         "instead of the autotuner's choice (for profiler runs, whose timings would mislead it)")
    ap.add_argument("--sweep-rows", type=int, default=0,
                    help="persistent IC-GN: subset rows per sweep tile (0 library default, -1 C order)")
    ap.add_argument("--icgn-staged", action="store_true",
                    help="pin the batched IC-GN kernels to the lean 4-warp sweep staged through TMA copies of g")
    ap.add_argument("--node-order", default="morton", choices=["morton", "index"],
                    help="persistent IC-GN work queue order")
    ap.add_argument("--no-quads", action="store_true", help="persistent IC-GN samples g itself, not its quad copy")
    ap.add_argument("--edge", type=int, default=512, help="--stage tiled: box edge target (tile_local)")
    ap.add_argument("--ncc-engine", default="auto", choices=["auto", "tiled", "fft", "fft_cluster", "plain"],
                    help="--stage pass: the integer search's engine")
    ap.add_argument("--frames", type=int, default=4, help="--stage series: deformed frames of the series")
    ap.add_argument("--stage", default="full", choices=["full", "pass", "ncc", "precompute", "tiled", "series"],
                    help="full: the benchmark line; pass / ncc / precompute: timing of one stage on a profiling case "
                         "(human-readable lines, no JSON), see stage_main")
    ap.add_argument("--shape", type=int, nargs=3, default=None, help="volume (nz ny nx) of a --stage case")
    ap.add_argument("--engine", type=int, default=2, help="--stage ncc: 0 tiled, 1 plain, 2 FFT, 3 FFT with Stockham")
    ap.add_argument("--half", type=int, default=8, help="--stage ncc: template half-width")
    ap.add_argument("--radius", type=int, default=16, help="--stage ncc: search radius")
    ap.add_argument("--per-node", action="store_true", help="--stage precompute: also time the per-node kernel")
    return ap.parse_args()


# --------------------------------------------------------------------------- profiling cases
def stage_main(args) -> None:
    """Timing of one stage on a seeded case small enough for a profiler capture; prints each repetition's wall
    time after a device synchronisation and the library's CUDA-event kernel times of the last repetition.

    pass        the configuration's whole pass (its parameters; --icgn-threads pins the lean IC-GN form) on a
                device-rendered pair of --shape (default 200 384 384 for configuration 5) with the configuration's
                beads, noise and field; --warmup passes first, then --steps timed ones
    ncc         the integer search (--engine, 2 FFT by default) on a 192^3 pair of Gaussian beads (0.03 / voxel,
                sigma 1.5, rendered on the device) moved by (1.3, -2.4, 3.1), a (2 --half + 1)^3 template at
                +- --radius (default 17^3 at +-16: the 1024 x 1024 x 306 workload's geometry), nodes every 12 voxels
    precompute  the separable precompute on a 306 x 512 x 512 volume (--shape) of 0.005 / voxel sigma-2 beads, 33^3
                subsets every 12 voxels (f and three gradients 1.28 GB, larger than L2); --per-node also times the
                per-node kernel and prints the largest relative difference of H between the forms
    tiled       the configuration's pass (full size unless --shape) resident on the device, then tiled.run_pass_tiled
                from host copies of the same frames with boxes of --edge voxels, once keeping the local boxes between
                stages and once streaming every box again; prints the boxes, the bytes uploaded and the largest
                difference to the resident result
    series      --frames single passes of the configuration's pair from pinned host memory (copies timed), then
                frames.run_series over frame 0 and the deformed frame repeated --frames times from host memory,
                accumulative (one prepared reference) and incremental (a new reference every frame)"""
    import torch

    from pyaldvc_b200 import configs
    from pyaldvc_b200 import kernels as K
    from pyaldvc_b200 import synthetic as S
    from pyaldvc_b200.mesh import build_grid_axes, grid_coords

    def timed(label, fn, n, unit_name):
        out = None
        for i in range(max(1, args.steps)):
            if i == max(1, args.steps) - 1:
                K.kernel_timing(True)
            torch.cuda.synchronize()
            t = time.time()
            out = fn()
            torch.cuda.synchronize()
            dt = time.time() - t
            print(f"{label} rep {i}: {1e3 * dt:.2f} ms, {1e6 * dt / n:.3f} us per {unit_name} ({n} {unit_name}s)", flush=True)
        print({k: (round(v[0], 3), v[1]) for k, v in K.kernel_timing_read().items()}, flush=True)
        K.kernel_timing(False)
        return out

    if args.stage == "pass":
        from pyaldvc_b200.pipeline import run_pass

        cfg = args.config
        shape = tuple(args.shape) if args.shape else (200, 384, 384)
        p = configs.params(cfg, icgn_sweep_rows=args.sweep_rows, icgn_node_order=args.node_order,
                                icgn_quads=not args.no_quads, ncc_engine=args.ncc_engine)
        if args.icgn_threads:
            p.threads, p.brick_floats = args.icgn_threads, 0
        if args.icgn_staged:
            p.threads, p.brick_floats = 128, -1
        f, g, mask, _ = configs.device_pair(cfg, shape=shape)
        for _ in range(args.warmup):
            run_pass(f, g, p, mask)
        res = timed(f"config {cfg} pass on {shape}", lambda: run_pass(f, g, p, mask), 1, "pass")
        it3 = [float(t.double().mean()) for t in getattr(res, "icgn3_iters", [])]
        print(f"{int(res.coords.shape[0])} nodes, mean 12-DOF iterations {float(res.n_iter_local.double().mean()):.3f}, "
              f"mean 3-DOF iterations per pass {[round(v, 3) for v in it3]}")
        return
    if args.stage == "tiled":
        from pyaldvc_b200 import pipeline as PL
        from pyaldvc_b200.pipeline import run_pass
        from pyaldvc_b200.tiling import run_pass_tiled

        cfg = args.config
        shape = tuple(args.shape) if args.shape else None
        p = configs.params(cfg)  # the autotuner's launch shapes, shared by both passes
        fd, gd, md, _ = configs.device_pair(cfg, shape=shape)
        f, g = fd.cpu().numpy(), gd.cpu().numpy()
        mask = None if md is None else md.cpu().numpy()
        n_vox = f.size
        for _ in range(args.warmup):
            whole = run_pass(fd, gd, p, md)
        whole = timed(f"config {cfg} resident pass on {f.shape}", lambda: run_pass(fd, gd, p, md), 1, "pass")
        del fd, gd, md
        torch.cuda.empty_cache()
        print("resident stages (ms)", {k: round(1e3 * v, 1) for k, v in whole.tracer.stages().items()}, flush=True)
        torch.cuda.empty_cache()
        for cache in (0, None):
            label = "kept boxes" if cache is None else "no box cache"
            res = timed(f"config {cfg} tiled pass, edge {args.edge}, {label}",
                        lambda: run_pass_tiled(f, g, p, mask=mask, edge=args.edge, cache_bytes=cache,
                                               tracer=PL.Tracer(sync=True)), 1, "pass")
            print("  stages (ms)", {k: round(1e3 * v, 1) for k, v in res.tracer.stages().items()}, flush=True)
            fr = res.frames
            du = float((res.U - whole.U).abs().max())
            st = {k: (v["boxes"], v["max_voxels"], v["retried"]) for k, v in res.tiles.stages.items()}
            print(f"  boxes (count, largest voxels, retried) {st}; {fr.bytes_uploaded / 1e9:.2f} GB uploaded "
                  f"({fr.bytes_uploaded / (n_vox * f.itemsize):.2f} x the pair), {fr.boxes_loaded} boxes built, "
                  f"{fr.cache_hits} cache hits; max |U - resident U| {du:.2e}; status equal "
                  f"{bool((res.status == whole.status).all())}", flush=True)
            del res, fr
            torch.cuda.empty_cache()
        return
    if args.stage == "series":
        from pyaldvc_b200.frames import run_series
        from pyaldvc_b200.pipeline import run_pass

        cfg = args.config
        shape = tuple(args.shape) if args.shape else None
        p = configs.params(cfg)
        fd, gd, md, _ = configs.device_pair(cfg, shape=shape)
        host = [fd.cpu().numpy()] + [gd.cpu().numpy()] * args.frames  # frame 0, then the deformed frame repeated
        masks = None if md is None else [md.cpu().numpy()] + [None] * args.frames
        n_nodes = None
        for _ in range(args.warmup):
            r = run_pass(fd, gd, p, md)
            n_nodes = int(r.coords.shape[0])
        del fd, gd, md
        torch.cuda.empty_cache()
        f_h = torch.from_numpy(host[0]).pin_memory()
        g_h = torch.from_numpy(host[1]).pin_memory()
        m_h = None if masks is None else torch.from_numpy(masks[0]).pin_memory()
        torch.cuda.synchronize()
        t = time.time()
        for _ in range(args.frames):  # single passes from pinned host memory, copies in the timed region
            r = run_pass(f_h.to("cuda", non_blocking=True), g_h.to("cuda", non_blocking=True), p,
                         None if m_h is None else m_h.to("cuda", non_blocking=True))
            r.U.cpu()
        torch.cuda.synchronize()
        single = time.time() - t
        print(f"config {cfg}: {args.frames} single passes from host memory {1e3 * single:.1f} ms "
              f"({1e3 * single / args.frames:.1f} ms per frame, {n_nodes * args.frames / single:.0f} nodes/s)", flush=True)
        for mode in ("accumulative", "incremental"):
            for rep in range(2):
                torch.cuda.synchronize()
                t = time.time()
                res = run_series(host, p, masks=masks, reference_mode=mode)
                torch.cuda.synchronize()
                dt = time.time() - t
            tm = res.timings
            print(f"config {cfg}: {mode} series of {args.frames} frames {1e3 * dt:.1f} ms ({1e3 * dt / args.frames:.1f} ms per frame, "
                  f"{n_nodes * args.frames / dt:.0f} nodes/s); references prepared in {1e3 * tm.get('reference_prepare', 0):.1f} ms, "
                  f"cumulative {1e3 * tm['cumulative']:.1f} ms, {tm['h2d_bytes'] / 1e9:.2f} GB uploaded; frames (s) "
                  f"{[round(fr.seconds, 3) for fr in res.frames]}", flush=True)
        return
    if args.stage == "ncc":
        n, h, r = 192, args.half, args.radius
        shape = (n, n, n)
        c, pk = S.draw_beads(shape, 0.03, 5)
        vols = []
        for cc in (c, S.displace_beads(c, S.translation((1.3, -2.4, 3.1)))):
            acc = torch.zeros(shape, dtype=torch.float64, device="cuda")
            K.render_beads(acc, cc, pk, 1.5, 6)
            vols.append(acc.float().contiguous())
            del acc
        f, g = vols
        m = h + r + 2
        ax = np.arange(m, n - m, 12)
        zz, yy, xx = np.meshgrid(ax, ax, ax, indexing="ij")
        coords = np.stack([xx.ravel(), yy.ravel(), zz.ravel()], 1).astype(np.int64)
        for _ in range(args.warmup):
            K.ncc_search(f, g, coords, (h, h, h), (r, r, r), None, args.engine)
        timed(f"engine {args.engine}", lambda: K.ncc_search(f, g, coords, (h, h, h), (r, r, r), None, args.engine), len(coords),
              "node")
        return
    if args.stage == "precompute":
        shape = tuple(args.shape) if args.shape else (306, 512, 512)
        c, pk = S.draw_beads(shape, 0.005, 7)
        acc = torch.zeros(shape, dtype=torch.float64, device="cuda")
        K.render_beads(acc, c, pk, 2.0, 8)
        f = K.normalize(acc.float().contiguous())
        del acc
        gx, gy, gz = K.gradients(f)
        w = (32, 32, 32)
        x0, y0, z0 = build_grid_axes(shape, w, (12, 12, 12))
        axes = [np.round(np.asarray(a_)).astype(np.int64) for a_ in (x0, y0, z0)]
        half = (16, 16, 16)
        n = int(np.prod([len(a_) for a_ in axes]))
        for _ in range(args.warmup):
            K.precompute_grid(*axes, half, f, gx, gy, gz, 0.5, 1e12)
        Hg = timed("grid form", lambda: K.precompute_grid(*axes, half, f, gx, gy, gz, 0.5, 1e12)[0], n, "node")
        if args.per_node:
            coords = torch.from_numpy(np.round(grid_coords(x0, y0, z0)).astype(np.int64)).cuda()
            Hp = timed("per-node form", lambda: K.precompute(coords, half, f, gx, gy, gz, None, 0.5, 1e12)[0], n, "node")
            print(f"max |dH| / max |H| = {float((Hg - Hp).abs().max() / Hp.abs().max()):.2e}", flush=True)
        return


# --------------------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi clock / throttle samples every 200 ms while running."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (OSError, ValueError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) == 7:
                self.rows.append(parts)

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}

        def num(x):
            try:
                return float(x)
            except ValueError:
                return float("nan")

        sm = np.array([num(r[0]) for r in self.rows])
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if r[3 + i].lower() == "active"})
        return {"sm_mhz": float(np.nanmedian(sm)), "sm_max_mhz": num(self.rows[0][1]), "power_w_max":
                float(np.nanmax([num(r[2]) for r in self.rows])), "reasons": reasons, "samples": len(self.rows)}


# --------------------------------------------------------------------------- CPU baseline (oracle, FP64)
def node_block(mesh_shape, edge: int):
    """(flat indices, block grid shape) of an edge^3 block of nodes at the centre of the node grid."""
    nz, ny, nx = mesh_shape
    e = [min(edge, s) for s in (nz, ny, nx)]
    st = [(s - k) // 2 for s, k in zip((nz, ny, nx), e)]
    iz, iy, ix = np.meshgrid(*[np.arange(a, a + k) for a, k in zip(st, e)], indexing="ij")
    return (iz * ny * nx + iy * nx + ix).ravel(), tuple(e)


def sample_box(c, spec: dict, vol_shape):
    """The volume box ((z0, z1), (y0, y1), (x0, x1)) a block of nodes ``c`` (M, 3) [x, y, z] reads: subsets with room
    for the displacement, and the NCC windows at the stated radius."""
    half = [int(w) // 2 for w in spec["winsize"]]
    h0 = [min(int(w), 16) // 2 for w in spec["winsize"]]
    reach = np.array([max(h + 16, a + r) + 8 for h, a, r in zip(half, h0, spec["search_radius"])])
    lo = np.maximum(c.min(axis=0) - reach, 0)
    hi = np.minimum(c.max(axis=0) + reach + 1, [vol_shape[2], vol_shape[1], vol_shape[0]])
    return ((int(lo[2]), int(hi[2])), (int(lo[1]), int(hi[1])), (int(lo[0]), int(hi[0])))


def oracle_prm(spec: dict) -> dict:
    """The oracle pass's parameters of a configuration (no early stop where the configuration runs without it)."""
    prm = {k: spec[k] for k in ("winsize", "search_radius", "interp_method") if k in spec}
    prm["use_global_step"] = spec.get("use_global_step", True)
    for k in ("mu", "beta", "admm_max_iter"):
        if k in spec:
            prm[k] = spec[k]
    if not spec.get("admm_early_stop", True):
        prm["admm_tol"] = -1.0
    return prm


def cpu_pass_sample(fn, gn, c_local, c_global, block_grid, spec: dict, mask, threads: int):
    """One AL-DVC pass of the FP64 oracle (the reference's CPU path restated: NCC with the reference's
    engine switch, FFT above 3e7 products, and radius expansion; precompute; 12-DOF with outlier filling; global
    step; ADMM) over a block of nodes as its own node grid, on normalised host volumes of the box the block reads.
    Returns (seconds, nodes, result)."""
    from oracle import oracle as orc

    orc.set_num_threads(threads)
    node_half = None
    if spec.get("node_winsize") is not None:
        node_half = np.asarray(spec["node_winsize"](c_global), dtype=np.int64) // 2
    spacing = tuple(float(s) for s in spec["winstepsize"])
    t0 = time.perf_counter()
    out = orc.aldvc_pass(fn, gn, c_local, block_grid, spacing, mask=None if mask is None else mask != 0, node_half=node_half,
                         **oracle_prm(spec))
    return time.perf_counter() - t0, int(c_local.shape[0]), out


def oracle_local_rms(fn, gn, c_local, spec: dict, mask, U0, P_gpu, st_gpu, c_global) -> float | None:
    """RMS difference of the device's raw 12-DOF displacements from the FP64 oracle's 12-DOF solve started at the
    same initial guess, on the nodes both converged (per subset shape, as the reference calls its kernels)."""
    from oracle import oracle as orc

    n = c_local.shape[0]
    half = tuple(int(w) // 2 for w in spec["winsize"])
    halves = (np.tile(np.asarray(half), (n, 1)) if spec.get("node_winsize") is None
              else np.asarray(spec["node_winsize"](c_global), dtype=np.int64) // 2)
    mode = {"linear": 0, "cubic": 1, "bspline": 2}[spec["interp_method"]]
    gx, gy, gz = orc.compute_gradients(fn)
    m = np.ones((1, 1, 1), np.uint8) if mask is None else np.ascontiguousarray(mask, dtype=np.uint8)
    P = np.full((n, 12), np.nan)
    st = np.full(n, -1, dtype=np.int8)
    for sh in np.unique(halves, axis=0):
        sel = np.flatnonzero((halves == sh).all(axis=1))
        hs = tuple(int(v) for v in sh)
        H, L, mf, bf, _, valid = orc.precompute_nodes(c_local[sel], *hs, fn, gx, gy, gz, m, 0.5, 1e12, 1)
        P0 = np.zeros((len(sel), 12))
        P0[:, 9:] = U0[sel]
        P[sel], _, st[sel], _ = orc.icgn_12dof_parallel(c_local[sel], P0, *hs, fn, gx, gy, gz, m, gn, mode, L, mf, bf, valid, 1e-2,
                                                        1e-3, 100, 5, 1)
    ok = (st == 0) & (st_gpu == 0)
    if not ok.any():
        return None
    d = P_gpu[ok, 9:] - P[ok, 9:]
    return float(np.sqrt(np.mean(d * d)))


def run_reference(args):
    """CPU arm: the FP64 oracle restatement of the reference's CPU path (the reference is Python/Numba with no
    compiled code to build) on the host cores, one bounded sample of the workload per step: a block of nodes of the
    configuration's node grid, run as its own grid through the whole pass, on that block's box of the volume pair
    rendered on the host.  Uses neither the device nor this package's CUDA library."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import oracle as orc
    from pyaldvc_b200 import configs, mesh

    spec = configs.spec(args.config)
    shape = configs.shape_of(args.config)
    x0, y0, z0 = mesh.build_grid_axes(shape, spec["winsize"], spec["winstepsize"])
    coords = np.round(mesh.grid_coords(x0, y0, z0)).astype(np.int64)
    grid_shape = (len(z0), len(y0), len(x0))
    block, block_grid = node_block(grid_shape, args.cpu_nodes)
    c = coords[block]
    box = sample_box(c, spec, shape)
    f_raw, g_raw, mask = configs.host_box(args.config, box)
    fn, gn = orc.normalize_volume(f_raw), orc.normalize_volume(g_raw)
    c_local = c - np.array([box[2][0], box[1][0], box[0][0]], dtype=np.int64)[None, :]
    threads = os.cpu_count() or 1
    small, small_grid = node_block(block_grid, 2)
    for _ in range(max(0, min(args.warmup, 1))):  # the first call builds the oracle library and warms its code paths
        cpu_pass_sample(fn, gn, c_local.reshape(block_grid + (3,))[tuple(slice(0, k) for k in small_grid)].reshape(-1, 3),
                        c.reshape(block_grid + (3,))[tuple(slice(0, k) for k in small_grid)].reshape(-1, 3), small_grid, spec,
                        mask, threads)
    times = []
    n = 0
    engine = orc.ncc_engine(tuple(min(int(w), 16) // 2 for w in spec["winsize"]), spec["search_radius"])
    for _ in range(args.steps):
        dt, n, _ = cpu_pass_sample(fn, gn, c_local, c, block_grid, spec, mask, threads)
        times.append(dt)
    value = n / float(np.mean(times))
    sample = (f"{n} nodes ({'x'.join(str(k) for k in block_grid)} block at the grid centre, run as its own node grid) "
              f"per step through the whole pass (NCC on the {engine} engine with expansion, precompute, 12-DOF with filling"
              f"{', global step and ADMM' if spec.get('use_global_step', True) else ''}), FP64 oracle, {threads} threads, "
              f"on a {'x'.join(str(b[1] - b[0]) for b in box)} box of the pair rendered on the host")
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": "nodes/s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * float(np.mean(times)), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD[args.config], "config_index": args.config, "nodes_per_step": n},
        "cpu_baseline": {"value": value, "unit": "nodes/s", "cores": threads, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": "nodes/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


HBM_FALLBACK_GBS = 6650.0


def _peaks() -> dict:
    """Peaks for the roofline.  The hot kernels are FP32 CUDA-core bound; the measured-peaks file holds HBM and
    bf16 tensor figures only, so the FP32 peak is the nominal rate of the device (SMs x 128 FP32 lanes x 2 x max clock)."""
    import torch

    props = torch.cuda.get_device_properties(0)
    mhz = 1965.0
    path = os.path.join(REPO, "MEASURED_PEAKS.json")
    hbm = None
    if os.path.exists(path):
        with open(path) as fh:
            mp = json.load(fh)
        mhz = float(mp.get("sm_max_mhz", mhz))
        hbm = mp.get("hbm_gbs")
    hbm_source = "measured (MEASURED_PEAKS.json hbm_gbs)"
    if hbm is None:  # no measured-peaks file on this box: the earlier copy-bandwidth measurement of this GPU pool
        hbm = HBM_FALLBACK_GBS
        hbm_source = "fallback: 6650 GB/s, an earlier STREAM-style copy measurement on B200s of this pool"
    fp32 = props.multi_processor_count * 128 * 2 * mhz * 1e6 / 1e12
    return {"fp32_tflops": fp32, "hbm_gbs": hbm, "hbm_source": hbm_source,
            "fp32_source": f"nominal FP32 CUDA-core rate: {props.multi_processor_count} SMs x 128 lanes x 2 flop x {mhz:.0f} MHz"}


def _smooth_len(n: int) -> int:
    m = int(n)
    while True:
        k = m
        for q in (2, 3, 5):
            while k % q == 0:
                k //= q
        if k == 1:
            return m
        m += 1


FFT_REG_SIZES = (36, 40, 48, 50, 54, 60, 64)  # cubic FFT boxes transformed a line per thread in registers

# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) per unit of work of the dominant kernels, from ncu captures
# of the 1024 x 1024 x 306 workload's kernels on a 200 x 384 x 384 box of the same beads, field and parameters (11,774
# nodes; profiles/ncu_icgn_lean_config5_box.md, profiles/dram_config5_box.md), scaled here by the units a launch of
# the measured pass processes.  Units: node-iterations for IC-GN, nodes for the NCC kernels.
TRAFFIC_PER_UNIT = {
    "icgn12_lean": ("node-iteration", (4.409e9 + 0.687e9) / (11774 * 2.237)),
    "icgn3_lean": ("node-iteration", (5.129e9 + 0.274e9) / (11774 * 1.241)),
    "fft_pass1": ("node", 787.09e6 / 811),
    "fft_pass2": ("node", 958.01e6 / 811),
    "fft_pass3": ("node", 367.63e6 / 811),
    "ncc_peak": ("node", 165.55e6 / (512 * 2**20 // (33**3 * 4))),
}
# issue-slot, L1 and FMA-pipe utilisation of the IC-GN kernels (ncu on the same box): the FP32 roof is not what bounds
# them; their sweeps are gathers through L1, so issue slots and L1 throughput are the roofs they run against
ICGN_NCU_BOX = {
    "icgn12_lean": {"issue_active": 0.563, "l1tex_throughput": 0.618, "fma_pipe": 0.362, "l1_hit": 0.802, "l2_hit": 0.855},
    "icgn3_lean": {"issue_active": 0.626, "l1tex_throughput": 0.789, "fma_pipe": 0.367, "l1_hit": 0.767, "l2_hit": 0.805},
}


def _kernel_roofline(ktimes: dict, res, p, vol_shape, peaks) -> dict:
    """Roofline of every timed kernel of one pass: algorithmic work of the pass for that kernel (bytes it must move,
    or FP32 flops) over its summed device time.  Work per unit:
      fft_pass1  window + template in, spectrum planes out: (wz wy wx + sz sy sxp) 4 B + wz Ny Nx 8 B per node
      fft_pass2  spectrum planes in, product planes out: (wz Ny + vz Ny') Nx 8 B per node
      fft_pass3  product planes in, box sums in, map out: vz Ny' Nx 8 B + 3 n_off 4 B per node
                 (Ny' = Ny / 2 + 1 for the in-register cubic boxes, which keep the product's Hermitian half; else Ny)
      ncc_peak   two sweeps of the FP32 map: 2 n_off 4 B per node; with the in-register FFT engine, whose pass 3 leaves
                 per-block map partials, the partials (32 B per block) and one block of map planes
      ncc_template  template in, centred template out: (n_tpl + sz sy sxp) 4 B per node
      box_pass   16 B per voxel per launch
      ncc_tiled / ncc_map  2 n_tpl n_off flop per node (direct cross term)
      precompute 162 S flop per node (per-node form); separable grid form: 16 B per voxel + its two intermediate sum
                 volumes written and read (80 B per voxel row and node column, 304 B per plane and node)
      icgn12_* 263 (cubic) / 87 (linear) flop per voxel-iteration, icgn3_* 239 / 63."""
    nvox = float(np.prod(vol_shape))
    byte_work, flop_work = {}, {}
    for n, half, rad, engine in getattr(res, "ncc_calls", []):
        s_ = [2 * int(h) + 1 for h in half]
        v_ = [2 * int(r) + 1 for r in rad]
        w_ = [a + b - 1 for a, b in zip(s_, v_)]
        N = [_smooth_len(w) for w in w_]
        sxp = (s_[0] + 3) // 4 * 4
        n_tpl, n_off = float(np.prod(s_)), float(np.prod(v_))
        plane = N[0] * N[1] * 8.0  # Nx Ny complex
        reg = N[0] == N[1] == N[2] and N[0] in FFT_REG_SIZES
        pplane = N[0] * (N[1] // 2 + 1) * 8.0 if reg else plane  # product plane
        if engine == 2:
            byte_work["fft_pass1"] = byte_work.get("fft_pass1", 0.0) + n * ((w_[0] * w_[1] * w_[2] + s_[2] * s_[1] * sxp) * 4.0 + w_[2] * plane)
            byte_work["fft_pass2"] = byte_work.get("fft_pass2", 0.0) + n * (w_[2] * plane + v_[2] * pplane)
            byte_work["fft_pass3"] = byte_work.get("fft_pass3", 0.0) + n * (v_[2] * pplane + 3.0 * n_off * 4.0)
        if engine in (0, 2):
            byte_work["ncc_template"] = byte_work.get("ncc_template", 0.0) + n * (n_tpl + s_[2] * s_[1] * sxp) * 4.0
        if engine == 0:
            flop_work["ncc_tiled"] = flop_work.get("ncc_tiled", 0.0) + n * 2.0 * n_tpl * n_off
        if engine == 1:
            flop_work["ncc_map"] = flop_work.get("ncc_map", 0.0) + n * 2.0 * n_tpl * n_off
        if engine == 2 and reg:
            nh = N[1] // 2 + 1
            p3 = max(1, min(70000 // (N[0] * (nh | 1) * 8), 256 // nh))  # map planes per pass-3 block
            peak_b = -(-v_[2] // p3) * 32.0 + min(p3, v_[2]) * v_[1] * v_[0] * 4.0
        else:
            peak_b = 2.0 * n_off * 4.0
        byte_work["ncc_peak"] = byte_work.get("ncc_peak", 0.0) + n * peak_b
    if "box_pass" in ktimes:
        byte_work["box_pass"] = ktimes["box_pass"][1] * 16.0 * nvox
    half = [int(w) // 2 for w in p.winsize]
    if getattr(res, "node_half", None) is not None:
        S_node = ((2 * res.node_half.double() + 1).prod(dim=1)).cpu().numpy()
    else:
        S_node = np.full(res.coords.shape[0], float(np.prod([(2 * h) // p.subset_stride + 1 for h in half])))
    c12, c3 = (87.0, 63.0) if p.interp_method == "linear" else (263.0, 239.0)
    if getattr(res, "precompute_form", "per_node") == "grid":
        # separable form: f, gx, gy, gz read once (16 B / voxel), the x pass's 20 FP32 row sums per (z, y, node column)
        # written and read, the y pass's 38 FP64 sums per (z, node row, node column) written and read
        gz_, gy_, gx_ = res.grid_shape
        nz_, ny_ = vol_shape[0], vol_shape[1]
        byte_work["precompute"] = 16.0 * nvox + 2 * 80.0 * nz_ * ny_ * gx_ + 2 * 304.0 * nz_ * gy_ * gx_
    else:
        flop_work["precompute"] = 162.0 * float(S_node.sum())
    it12 = getattr(res, "n_iter_local", res.n_iter).cpu().numpy().astype(np.float64)
    it3 = sum((t.cpu().numpy().astype(np.float64) for t in getattr(res, "icgn3_iters", [])), np.zeros_like(it12))
    for form in ("lean", "batched", "plain"):
        flop_work[f"icgn12_{form}"] = c12 * float((it12 * S_node).sum())
        flop_work[f"icgn3_{form}"] = c3 * float((it3 * S_node).sum())
    # units of the measured pass for the traffic scaling
    units = {"icgn12_lean": float(it12.sum()), "icgn3_lean": float(it3.sum())}
    fft_nodes = float(sum(n for n, _, _, e in getattr(res, "ncc_calls", []) if e == 2))
    for k in ("fft_pass1", "fft_pass2", "fft_pass3"):
        units[k] = fft_nodes
    units["ncc_peak"] = float(sum(n for n, _, _, _ in getattr(res, "ncc_calls", [])))
    total_ms = sum(ms for ms, _ in ktimes.values())
    out = {}
    for name, (ms, launches) in ktimes.items():
        row = {"ms": ms, "launches": launches, "ms_share": ms / total_ms if total_ms else None}
        traffic = None
        if name in TRAFFIC_PER_UNIT and units.get(name):
            traffic = TRAFFIC_PER_UNIT[name][1] * units[name] / max(1, launches)  # bytes per launch
        if name in byte_work and peaks.get("hbm_gbs"):
            ach = byte_work[name] / (ms / 1e3) / 1e9
            row.update({"bound": "hbm", "achieved": ach, "peak": peaks["hbm_gbs"], "unit": "GB/s", "frac": ach / peaks["hbm_gbs"],
                        "traffic": traffic, "peak_source": peaks["hbm_source"]})
            if traffic is not None:
                row["traffic_over_work"] = traffic * max(1, launches) / byte_work[name]
        elif name in flop_work:
            ach = flop_work[name] / (ms / 1e3) / 1e12
            row.update({"bound": "fp32", "achieved": ach, "peak": peaks["fp32_tflops"], "unit": "TFLOP/s",
                        "frac": ach / peaks["fp32_tflops"], "traffic": traffic, "peak_source": peaks["fp32_source"]})
            if traffic is not None:
                row["dram_gbs"] = traffic * max(1, launches) / (ms / 1e3) / 1e9
            if name in ICGN_NCU_BOX:
                box = ICGN_NCU_BOX[name]
                row["ncu_box"] = box
                # the roofs the kernel runs against, as fractions: FP32 from this run; issue slots and L1/TEX throughput
                # from the box capture (the gather's L1 wavefronts and the sweep's instruction count bind it)
                row["roofs"] = {"fp32": row["frac"], "issue_slots": box["issue_active"], "l1tex": box["l1tex_throughput"]}
                row["binding_roof"] = max(row["roofs"], key=row["roofs"].get)
        if traffic is not None:
            row["traffic_source"] = "ncu DRAM bytes per " + TRAFFIC_PER_UNIT[name][0] + " on the 200x384x384 box, scaled"
        out[name] = row
    return out


# --------------------------------------------------------------------------- B200 arm
def _tuned_shapes() -> list:
    """The autotuner's choice of (threads, brick_floats) per IC-GN kernel and its timings (ms per sample launch)."""
    from pyaldvc_b200 import autotune

    rows = []
    for k, choice in autotune._cache.items():
        t = autotune.timings(k) or {}
        rows.append({"ndof": k[0], "mode": k[1], "half": list(k[3]), "choice": list(choice),
                     "ms": {f"{a}x{b}": round(v, 3) for (a, b), v in t.items()}})
    return rows


def run_znssd(args):
    """Differentiation workload: ZNSSD cost of 10,000 warped 21^3 subsets of a 192^3 bead pair and its gradient
    with respect to the 12 warp parameters and the deformed volume, through the torch.autograd.Function.  A step
    is one forward + backward over all subsets; value = subsets per second.  The CPU baseline is the FP64 oracle
    forward plus a fourth-order central-difference gradient (48 more forward evaluations) on a 64-subset sample."""
    import torch

    from oracle import oracle as O
    from pyaldvc_b200 import kernels as K
    from pyaldvc_b200 import synthetic as S
    from pyaldvc_b200.znssd import znssd

    shape, n, h = (192, 192, 192), 10000, 10
    c, pk = S.draw_beads(shape, 0.02, 4)
    rng = np.random.default_rng(4)
    f = S.render_beads(shape, c, pk, 1.5) + rng.normal(0.0, 0.01, shape).astype(np.float32)
    g = S.render_beads(shape, S.displace_beads(c, S.translation((0.6, -0.9, 1.2))), pk, 1.5) + rng.normal(0.0, 0.01, shape).astype(np.float32)
    f, g = S.normalize_volume(f), S.normalize_volume(g)
    coords = rng.integers(h + 6, 192 - h - 6, size=(n, 3)).astype(np.int64)
    P = np.zeros((n, 12))
    P[:, :9] = rng.uniform(-0.03, 0.03, size=(n, 9))
    P[:, 9:] = rng.uniform(-2.0, 2.0, size=(n, 3))
    fd_, gd_ = torch.from_numpy(f).cuda(), torch.from_numpy(g).cuda()
    cd, Pd = torch.from_numpy(coords).cuda(), torch.from_numpy(P).cuda()
    w = torch.ones(n, dtype=torch.float64, device="cuda")

    def step():
        Pt = Pd.clone().requires_grad_(True)
        gt = gd_.clone().requires_grad_(True)
        cost = znssd(Pt, gt, fd_, cd, (h, h, h), "cubic")
        (cost * w).sum().backward()
        return cost, Pt.grad, gt.grad

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    lib = K.lib()
    l0 = lib.aldvc_launch_count()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(0) as clocks:
        e0.record()
        for _ in range(args.steps):
            cost, gP, gG = step()
        e1.record()
        torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    launches = (lib.aldvc_launch_count() - l0) / args.steps
    # accuracy on a sample: kernel gradient vs fourth-order central differences (h = 1e-3) of the FP64 oracle
    sel = np.arange(64)
    gps = gP.detach().cpu().numpy()[sel]
    fd4 = np.empty((len(sel), 12))
    t0 = time.perf_counter()
    base = O.znssd(f, g, coords[sel], P[sel], (h, h, h), 1)
    for k in range(12):
        cs = []
        for d in (1e-3, -1e-3, 2e-3, -2e-3):
            Q = P[sel].copy()
            Q[:, k] += d
            cs.append(O.znssd(f, g, coords[sel], Q, (h, h, h), 1))
        fd4[:, k] = (8.0 * (cs[0] - cs[1]) - (cs[2] - cs[3])) / 12e-3
    cpu_s = time.perf_counter() - t0
    rel = np.linalg.norm(gps - fd4, axis=1) / np.linalg.norm(fd4, axis=1)
    cost_ref = base
    cost_rel = float(np.max(np.abs(cost.detach().cpu().numpy()[sel] - cost_ref) / np.abs(cost_ref)))
    # algorithmic work: forward samples every voxel twice (64 taps) and backward once with its gradient
    # (64 taps x 4 accumulations) plus 64 scatter atomics; bytes = the subsets' f reads + 3 x 64 taps
    S_ = (2 * h + 1) ** 3
    flops = n * S_ * (2 * 2 * 64 + 2 * 4 * 64)
    out = {
        "metric": ZNSSD_METRIC, "value": n / (ms / 1e3), "unit": "subsets/s", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 interpolation, f64 residual and reductions", "data": "synthetic",
        "config": {"workload": WORKLOAD[4], "config_index": 4, "subsets": n, "subset": [2 * h + 1] * 3,
                   "l2": "volumes 28 MB each (inside L2); gradient volume rewritten every step"},
        "accuracy": {"grad_P_rel_vs_fd4_max": float(rel.max()), "grad_P_rel_vs_fd4_median": float(np.median(rel)),
                     "cost_rel_vs_fp64_oracle_max": cost_rel, "sample_subsets": len(sel)},
        "gpu_launches": int(round(launches)),
        "roofline": {"bound": "fp32", "achieved": flops / (ms / 1e3) / 1e12, "peak": 74.44992, "unit": "TFLOP/s",
                     "frac": flops / (ms / 1e3) / 1e12 / 74.44992, "traffic": None,
                     "peak_source": "nominal FP32 CUDA-core rate: 148 SMs x 128 lanes x 2 flop x 1965 MHz",
                     "work": "interpolation FMAs: forward 2 x 64 taps, backward 64 taps x 4 sums, per voxel"},
        "cpu_baseline": {"value": len(sel) / cpu_s, "unit": "subsets/s", "cores": O.num_threads(),
                         "kind": "port", "sample": "64 subsets: FP64 oracle forward + 4th-order central-difference gradient"},
        "clocks": clocks.summary(),
    }
    print(json.dumps(out), flush=True)


def max_over_ranks(x: float, world: int, device="cuda") -> float:
    """The largest value of ``x`` over the ranks (a device time: the slowest replica sets the job's time).  Every
    rank calls it at the same point; with one rank it returns ``x`` and makes no collective call."""
    if world <= 1:
        return float(x)
    import torch
    import torch.distributed as dist

    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def main():
    args = parse()
    if args.stage != "full":
        stage_main(args)
        return
    if args.impl == "reference" and args.config != 4:
        run_reference(args)
        return
    if args.config == 4:
        if int(os.environ.get("RANK", "0")) == 0:
            if args.impl == "reference":
                print(json.dumps({"impl": "reference", "unavailable": "the reference has no differentiable ZNSSD residual"}))
            else:
                run_znssd(args)
        return
    import torch
    import torch.distributed as dist

    from pyaldvc_b200 import configs
    from pyaldvc_b200 import kernels as K
    from pyaldvc_b200.cuda_kernels import cuda_available, unavailable_reason
    from pyaldvc_b200.pipeline import Tracer, run_pass

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=600), device_id=torch.device("cuda", local))
    if not cuda_available():
        raise RuntimeError(f"B200 library unusable: {unavailable_reason()}")

    cfg = args.config
    p = configs.params(cfg, icgn_sweep_rows=args.sweep_rows, icgn_node_order=args.node_order,
                                icgn_quads=not args.no_quads)
    if args.icgn_threads:
        p.threads, p.brick_floats = args.icgn_threads, 0
    if args.icgn_staged:
        p.threads, p.brick_floats = 128, -1
    f, g, mask, disp = configs.device_pair(cfg, seed=1000 + 17 * rank)
    torch.cuda.synchronize()

    def one_pass(variant=K.BATCHED, tracer=None):
        p.variant = variant
        return run_pass(f, g, p, mask, tracer=tracer)

    for _ in range(args.warmup):
        res = one_pass()
    torch.cuda.synchronize()

    # ---- timed region: K passes, inputs resident in HBM
    lib = K.lib()
    tracers = [Tracer() for _ in range(args.steps)]
    launches0 = lib.aldvc_launch_count()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clocks:
        ev0.record()
        for k in range(args.steps):
            res = one_pass(tracer=tracers[k])
        ev1.record()
        torch.cuda.synchronize()
    launches = (lib.aldvc_launch_count() - launches0) / args.steps
    if world > 1:
        dist.barrier()
    elapsed = ev0.elapsed_time(ev1) / 1e3
    elapsed_max = max_over_ranks(elapsed, world)
    n_nodes = int(res.coords.shape[0])
    value = world * n_nodes * args.steps / elapsed_max
    stages = {}
    for tr in tracers:
        for k_, v_ in tr.stages().items():
            stages[k_] = stages.get(k_, 0.0) + v_ / args.steps

    # accuracy against the ground-truth field (interior nodes that converged)
    coords = res.coords.cpu().numpy()
    U = res.U.cpu().numpy()
    U_local = res.P_local[:, 9:].cpu().numpy()
    status_local = res.status_local.cpu().numpy()
    truth = configs.truth_at(disp, coords)
    status = res.status.cpu().numpy()
    valid = res.valid.cpu().numpy()
    gs_ = res.grid_shape
    # interior = every node of the 3x3x3 neighbourhood valid (the grid border and an ROI's boundary layer excluded)
    vg = valid.reshape(gs_)
    interior = np.zeros(gs_, dtype=bool)
    interior[1:-1, 1:-1, 1:-1] = True
    for dz in (-1, 0, 1):
        for dy in (-1, 0, 1):
            for dx in (-1, 0, 1):
                interior[1:-1, 1:-1, 1:-1] &= vg[1 + dz:gs_[0] - 1 + dz, 1 + dy:gs_[1] - 1 + dy, 1 + dx:gs_[2] - 1 + dx]
    sel = interior.ravel() & valid & (status == 0)
    rms_truth = float(np.sqrt(np.mean((U[sel] - truth[sel]) ** 2))) if sel.any() else float("nan")
    sel_all = valid & (status == 0)
    rms_truth_all = float(np.sqrt(np.mean((U[sel_all] - truth[sel_all]) ** 2))) if sel_all.any() else float("nan")
    sel_l = sel_all & (status_local == 0)
    rms_local_truth = float(np.sqrt(np.mean((U_local[sel_l] - truth[sel_l]) ** 2))) if sel_l.any() else float("nan")

    # ---- per-kernel roofline: one more pass with the library's CUDA-event kernel timing on
    peaks = _peaks()
    K.kernel_timing(True)
    r_t = one_pass()
    torch.cuda.synchronize()
    ktimes = K.kernel_timing_read()
    K.kernel_timing(False)
    roof = _kernel_roofline(ktimes, r_t, p, f.shape, peaks)
    dominant = max(roof, key=lambda k_: roof[k_]["ms"]) if roof else None

    # ---- plain form of the same pass
    plain = None
    if args.plain_steps > 0:
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ptr = [Tracer() for _ in range(args.plain_steps)]
        e0.record()
        for k in range(args.plain_steps):
            res_p = one_pass(K.PLAIN, tracer=ptr[k])
        e1.record()
        torch.cuda.synchronize()
        pe = max_over_ranks(e0.elapsed_time(e1) / 1e3, world)
        pst = {}
        for tr in ptr:
            for k_, v_ in tr.stages().items():
                pst[k_] = pst.get(k_, 0.0) + v_ / args.plain_steps
        Up = res_p.U.cpu().numpy()
        plain = {"value": n_nodes * args.plain_steps / pe, "unit": "nodes/s", "ms_per_step": 1e3 * pe / args.plain_steps,
                 "stages_ms": {k_: 1e3 * v_ for k_, v_ in pst.items()},
                 "max_abs_dU_vs_batched": float(np.nanmax(np.abs(Up - U)))}
        p.variant = K.BATCHED

    # ---- end to end: host buffers through the public API, copies inside the timed region
    f_h = f.cpu().pin_memory()
    g_h = g.cpu().pin_memory()
    m_h = None if mask is None else mask.cpu().pin_memory()
    # one untimed pass from the same buffers: the first copies out of freshly pinned memory carry one-time costs
    run_pass(f_h, g_h, p, m_h).U.to("cpu")
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        r = run_pass(f_h, g_h, p, m_h)  # the pass copies its host inputs (the deformed one behind the reference's preparation)
        U_host = r.U.to("cpu")
    e1.record()
    torch.cuda.synchronize()
    e2e_t = max_over_ranks(e0.elapsed_time(e1) / 1e3, world)
    h2d = f_h.numel() * f_h.element_size() + g_h.numel() * g_h.element_size() + (0 if m_h is None else m_h.numel())
    d2h = U_host.numel() * U_host.element_size()
    e2e_val = world * n_nodes * args.steps / e2e_t

    # ---- CPU baseline: the FP64 oracle on a bounded node block of the same workload (rank 0, N = 1)
    cpu = None
    rms_oracle = None
    if rank == 0 and world == 1 and not args.no_cpu:
        from oracle import oracle as orc

        threads = os.cpu_count() or 1
        spec = configs.spec(cfg)
        block, block_grid = node_block(res.grid_shape, args.cpu_nodes)
        cb = coords[block]
        box = sample_box(cb, spec, tuple(f.shape))
        sl = tuple(slice(a_, b_) for a_, b_ in box)
        fn = np.ascontiguousarray(K.normalize(f)[sl].cpu().numpy())  # the device pass's own normalised volumes
        gn = np.ascontiguousarray(K.normalize(g)[sl].cpu().numpy())
        mb = None if mask is None else np.ascontiguousarray(mask[sl].cpu().numpy())
        c_local = cb - np.array([box[2][0], box[1][0], box[0][0]], dtype=np.int64)[None, :]
        dt, nb, _ = cpu_pass_sample(fn, gn, c_local, cb, block_grid, spec, mb, threads)
        engine = orc.ncc_engine(tuple(min(int(w), 16) // 2 for w in spec["winsize"]), spec["search_radius"])
        cpu = {"value": nb / dt, "unit": "nodes/s", "cores": threads, "kind": "port",
               "sample": f"{nb} nodes ({'x'.join(str(k) for k in block_grid)} block at the grid centre, run as its own node "
                         f"grid) through the whole pass (NCC on the {engine} engine with expansion, precompute, 12-DOF with "
                         f"filling{', global step and ADMM' if p.use_global_step else ''}), FP64 oracle"}
        U0_block = res.U0[block].cpu().numpy()
        rms_oracle = oracle_local_rms(fn, gn, c_local, spec, mb, U0_block, res.P_local[block].cpu().numpy(), status_local[block],
                                      cb)

    out = {
        "metric": METRIC, "value": value, "unit": "nodes/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * elapsed_max / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic",
        "config": {"workload": WORKLOAD[cfg], "config_index": cfg, "nodes_per_step": n_nodes, "volume_shape": list(f.shape),
                   "volume_dtype": str(f.dtype).replace("torch.", ""), "l2": "inputs larger than L2"
                   if f.numel() * f.element_size() > 126e6 else "inputs smaller than L2 (every pass rewrites its buffers)",
                   "parallelism": f"replica x{world}"},
        "stages_ms": {k_: 1e3 * v_ for k_, v_ in stages.items()},
        "accuracy": {"rms_vs_truth_vox": rms_truth, "nodes_scored": int(sel.sum()), "converged_frac": float(np.mean(status[valid] == 0)),
                     "rms_vs_truth_all_valid_vox": rms_truth_all, "rms_local_vs_truth_vox": rms_local_truth,
                     "rms_local_vs_fp64_oracle_vox": rms_oracle},
        "gpu_launches": int(round(launches)),
        "roofline": None if dominant is None else {k_: v_ for k_, v_ in roof[dominant].items() if k_ != "ms_share"} | {"kernel": dominant},
        "roofline_kernels": roof,
        "cpu_baseline": cpu,
        "plain": plain,
        "batched_over_plain": None if plain is None else value / world / plain["value"],
        "batched_over_plain_stages": None if plain is None else
        {k_: plain["stages_ms"][k_] / (1e3 * v_) for k_, v_ in stages.items() if k_ in plain["stages_ms"] and v_ > 0},
        "e2e": {"value": e2e_val, "unit": "nodes/s", "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h)},
        "clocks": clocks.summary(),
        "icgn_launch_shapes": _tuned_shapes(),
    }
    if rank == 0:
        print(json.dumps(out), flush=True)
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
