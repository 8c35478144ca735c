"""Timing of the two precompute forms on a seeded bead volume (a comparison tool for the forms).

    python -m pyaldvc_b200.precompute_probe [reps] [--shape NZ NY NX] [--winsize W] [--step S] [--per-node]

Defaults: 3 repetitions, a 306 x 512 x 512 volume (f and three stored gradients: 1.28 GB, larger than L2), 32^3
subsets every 12 voxels (the geometry of the 1024 x 1024 x 306 workload).  Prints each repetition's wall time after a
device synchronisation and the library's CUDA-event time of the precompute of the last one; ``--per-node`` also
times the per-node kernel and reports the largest relative difference of H between the forms.
"""

from __future__ import annotations

import argparse
import time

import numpy as np


def main(argv=None) -> None:
    import torch

    from . import kernels as K
    from . import synthetic as S
    from .mesh import build_grid_axes, grid_coords

    ap = argparse.ArgumentParser()
    ap.add_argument("reps", nargs="?", type=int, default=3)
    ap.add_argument("--shape", type=int, nargs=3, default=(306, 512, 512))
    ap.add_argument("--winsize", type=int, default=32)
    ap.add_argument("--step", type=int, default=12)
    ap.add_argument("--per-node", action="store_true")
    args = ap.parse_args(argv)
    shape = tuple(args.shape)
    c, pk = S.draw_beads(shape, 0.005, 7)
    acc = torch.zeros(shape, dtype=torch.float64, device="cuda")
    K.render_beads(acc, c, pk, 2.0, 8)
    f = K.normalize(acc.float().contiguous())
    del acc
    gx, gy, gz = K.gradients(f)
    w = (args.winsize,) * 3
    x0, y0, z0 = build_grid_axes(shape, w, (args.step,) * 3)
    axes = [np.round(np.asarray(a)).astype(np.int64) for a in (x0, y0, z0)]
    half = tuple(v // 2 for v in w)
    n = int(np.prod([len(a) for a in axes]))
    for i in range(args.reps):
        if i == args.reps - 1:
            K.kernel_timing(True)
        torch.cuda.synchronize()
        t = time.time()
        Hg = K.precompute_grid(*axes, half, f, gx, gy, gz, 0.5, 1e12)[0]
        torch.cuda.synchronize()
        dt = time.time() - t
        print(f"grid form rep {i}: {1e3 * dt:.2f} ms, {1e9 * dt / n:.1f} ns/node ({n} nodes)", flush=True)
    print({k: (round(v[0], 3), v[1]) for k, v in K.kernel_timing_read().items()})
    K.kernel_timing(False)
    if args.per_node:
        coords = torch.from_numpy(np.round(grid_coords(x0, y0, z0)).astype(np.int64)).cuda()
        torch.cuda.synchronize()
        t = time.time()
        Hp = K.precompute(coords, half, f, gx, gy, gz, None, 0.5, 1e12)[0]
        torch.cuda.synchronize()
        print(f"per-node form: {1e3 * (time.time() - t):.2f} ms; max |dH| / max |H| = "
              f"{float((Hg - Hp).abs().max() / Hp.abs().max()):.2e}", flush=True)


if __name__ == "__main__":
    main()
