"""Timing of the integer NCC search engines on a seeded bead pair (a comparison tool for the engines).

    python -m pyaldvc_b200.ncc_probe [engine] [reps] [--size N] [--half H] [--radius R]

engine: 0 tiled, 1 plain, 2 FFT, 3 FFT with Stockham transforms.  Defaults: FFT, 3 repetitions, a 192^3 pair,
a 17^3 template (half 8) and a +-16 search (the geometry of the 1024 x 1024 x 306 workload), nodes every 12 voxels.
Prints the wall time of each repetition after a device synchronisation, and the per-kernel device times of the
last one (the library's CUDA-event kernel timing).
"""

from __future__ import annotations

import argparse
import time

import numpy as np


def main(argv=None) -> None:
    import torch

    from . import kernels as K
    from . import synthetic as S

    ap = argparse.ArgumentParser()
    ap.add_argument("engine", nargs="?", type=int, default=2)
    ap.add_argument("reps", nargs="?", type=int, default=3)
    ap.add_argument("--size", type=int, default=192)
    ap.add_argument("--half", type=int, default=8)
    ap.add_argument("--radius", type=int, default=16)
    args = ap.parse_args(argv)
    n, h, r = args.size, args.half, args.radius
    shape = (n, n, n)
    c, pk = S.draw_beads(shape, 0.03, 5)
    vols = []
    for cc in (c, S.displace_beads(c, S.translation((1.3, -2.4, 3.1)))):  # rendered on the device (FP64 sums)
        acc = torch.zeros(shape, dtype=torch.float64, device="cuda")
        K.render_beads(acc, cc, pk, 1.5, 6)
        vols.append(acc.float().contiguous())
        del acc
    f, g = vols
    m = h + r + 2
    ax = np.arange(m, n - m, 12)
    zz, yy, xx = np.meshgrid(ax, ax, ax, indexing="ij")
    coords = np.stack([xx.ravel(), yy.ravel(), zz.ravel()], 1).astype(np.int64)
    for i in range(args.reps):
        if i == args.reps - 1:
            K.kernel_timing(True)
        torch.cuda.synchronize()
        t = time.time()
        K.ncc_search(f, g, coords, (h, h, h), (r, r, r), None, args.engine)
        torch.cuda.synchronize()
        dt = time.time() - t
        print(f"engine {args.engine} rep {i}: {1e3 * dt:.2f} ms, {1e6 * dt / len(coords):.2f} us/node ({len(coords)} nodes)", flush=True)
    print({k: (round(v[0], 3), v[1]) for k, v in K.kernel_timing_read().items()})
    K.kernel_timing(False)


if __name__ == "__main__":
    main()
