"""Launch-shape autotuner for the batched IC-GN kernels.

The batched solver has two persistent kernel forms:

* lean: 1, 2 or 4 warps per node (``threads`` 32/64/128); the deformed volume is sampled through L1,
  so up to 16 nodes share an SM and one node's FP64 control step hides behind the others' sampling;
* brick: 256 or 512 threads per node; the deformed subset is staged in shared memory in z-chunks
  that fit ``brick_floats`` floats;
* staged: the lean 4-warp sweep with each chunk's box of g brought into shared memory by TMA tensor copies
  (``(128, -1)``; cubic / B-spline with stored gradients and one subset shape, else it runs as the lean form).

Which is fastest depends on the subset size, the interpolation and the DOF count, so ``tune`` times
every candidate on a sample of the real nodes (CUDA events on the current stream, one untimed launch
first), keeps the fastest per key for the life of the process and returns ``(threads, brick_floats)``.
Inside a CUDA-graph capture nothing is timed: the cached choice, or the library default, is used.
"""

from __future__ import annotations

import torch

CANDIDATES = ((32, 0), (64, 0), (128, 0), (128, -1), (256, 24576), (256, 49152), (512, 24576), (512, 49152))
SAMPLE_NODES = 8 * 148 * 16  # enough work for every resident CTA of a B200 to take several nodes

_cache: dict = {}


def key(ndof: int, mode: int, stored: bool, half, stride: int, masked: bool, n_nodes: int) -> tuple:
    """Cache key: the kernel instantiation and subset geometry; node counts are bucketed by powers of 4."""
    bucket = 0
    n = int(n_nodes)
    while n >= 4:
        n //= 4
        bucket += 1
    return (int(ndof), int(mode), bool(stored), tuple(int(h) for h in half), int(stride), bool(masked), bucket)


def cached(k: tuple):
    return _cache.get(k)


def clear() -> None:
    _cache.clear()


def sample_index(n_nodes: int, device="cuda") -> torch.Tensor:
    """A fixed, evenly spread sample of node indices (every k-th node), at most ``SAMPLE_NODES``."""
    n = int(n_nodes)
    if n <= SAMPLE_NODES:
        return torch.arange(n, device=device)
    step = n / SAMPLE_NODES
    return (torch.arange(SAMPLE_NODES, device=device, dtype=torch.float64) * step).long()


def tune(k: tuple, run, candidates=CANDIDATES, reps: int = 2) -> tuple[int, int]:
    """Time ``run(threads, brick_floats)`` for every candidate; return and cache the fastest pair."""
    hit = _cache.get(k)
    if hit is not None:
        return hit
    if torch.cuda.is_current_stream_capturing():
        return (0, 0)
    times = {}
    stream = torch.cuda.current_stream()
    for th, br in candidates:
        run(th, br)  # untimed: kernel attributes, occupancy, caches
        t0 = torch.cuda.Event(enable_timing=True)
        t1 = torch.cuda.Event(enable_timing=True)
        t0.record(stream)
        for _ in range(reps):
            run(th, br)
        t1.record(stream)
        t1.synchronize()
        times[(th, br)] = t0.elapsed_time(t1) / reps
    best = min(times, key=times.get)
    _cache[k] = best
    _timings[k] = times
    return best


_timings: dict = {}


def timings(k: tuple) -> dict | None:
    """Per-candidate milliseconds measured for key ``k`` (for reports)."""
    return _timings.get(k)
