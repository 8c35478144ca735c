"""The five benchmark configurations: seeded synthetic bead volume pairs and their solver parameters.

1. 64^3 float32, 0.02 beads/voxel, sigma 1.5, peak U(0.5, 1), Gaussian noise 0.01; uniform translation
   (1.3, -0.7, 0.4); step 8, subsets 20^3, trilinear, direct NCC +-4; local IC-GN only.
2. 128^3 float32, same beads; 2 % uniaxial strain along z plus u_x = 0.5 sin(2 pi y / 64); step 6,
   subsets 24^3, NCC +-8, tricubic; local IC-GN only.
3. 256^3 uint16 (0-4095); 5 degree rotation about z plus 1 % hydrostatic strain; spherical ROI of radius
   110; step 8, uneven anisotropic subsets from 16x16x24 (ROI centre) to 32^3 (ROI edge), one persistent launch
   for every shape; ADMM with beta 1e-3, 3 iterations, captured as a CUDA graph.
5. 1024 x 1024 x 306 uint16, 0.005 beads/voxel, sigma 2, Poisson (1000 photons per unit peak) plus
   Gaussian noise; Boussinesq indentation u_z = -10.5 a^2 / (a^2 + r^2 + d^2), a = 80, plus a 0.3 voxel
   random-phase background; step 12, subsets 32^3, NCC +-16, tricubic, 3 ADMM iterations.

Volumes up to 256^3 are rendered with NumPy (deterministic, shared with the CPU oracle); the large one
is rendered on the device with ``aldvc_render_beads`` (FP64 accumulation, so the float32 result does not
depend on the order of the atomic sums).
"""

from __future__ import annotations

import numpy as np

from . import synthetic as syn


def spec(cfg: int) -> dict:
    """The solver parameters of a configuration as plain values (PassParams / DVCPara names).  Every
    configuration seeds IC-GN from one full-resolution NCC search of the stated radius, with no global
    phase-correlation pre-shift (the reference's defaults are the pyramid search and the pre-shift)."""
    common = dict(init_guess_method="ncc", global_shift=False)
    if cfg == 1:
        return dict(winsize=(20, 20, 20), winstepsize=(8, 8, 8), search_radius=(4, 4, 4), interp_method="linear",
                    use_global_step=False, **common)
    if cfg == 2:
        return dict(winsize=(24, 24, 24), winstepsize=(6, 6, 6), search_radius=(8, 8, 8), interp_method="cubic",
                    use_global_step=False, **common)
    if cfg == 3:
        return dict(winsize=(32, 32, 32), winstepsize=(8, 8, 8), search_radius=(8, 8, 8), interp_method="cubic", beta=1e-3,
                    mu=1e-3, admm_max_iter=3, admm_early_stop=False, graph=True, node_winsize=uneven_winsize, **common)
    if cfg == 5:
        return dict(winsize=(32, 32, 32), winstepsize=(12, 12, 12), search_radius=(16, 16, 16), interp_method="cubic",
                    beta=1e-3, mu=1e-3, admm_max_iter=3, **common)
    raise ValueError(f"no configuration {cfg}")


def params(cfg: int, **over):
    """PassParams of a configuration (``spec``), with ``over`` applied."""
    from .pipeline import PassParams

    p = PassParams(**spec(cfg))
    for k, v in over.items():
        setattr(p, k, v)
    return p


ROI_RADIUS = 110.0


def uneven_winsize(coords) -> np.ndarray:
    """Per-node window sizes of configuration 3: 16 x 16 x 24 at the centre of the spherical ROI, growing with the
    distance r from it to 32 x 32 x 32 at r = 110 (even sizes, (x, y, z) order)."""
    c = np.asarray(coords, dtype=np.float64)
    centre = (np.asarray(shape_of(3)[::-1], dtype=np.float64) - 1.0) / 2.0
    t = np.clip(np.linalg.norm(c - centre[None, :], axis=1) / ROI_RADIUS, 0.0, 1.0)
    wxy = 2 * np.round((16.0 + 16.0 * t) / 2.0)
    wz = 2 * np.round((24.0 + 8.0 * t) / 2.0)
    return np.stack([wxy, wxy, wz], 1).astype(np.int64)


def shape_of(cfg: int):
    return {1: (64, 64, 64), 2: (128, 128, 128), 3: (256, 256, 256), 5: (306, 1024, 1024)}[cfg]


def displacement(cfg: int, shape=None):
    """The configuration's displacement field (x, y, z) -> (u, v, w); ``shape`` (nz, ny, nx) places it on a volume
    of another size (centred the same way)."""
    shape = shape_of(cfg) if shape is None else tuple(shape)
    centre = tuple((s - 1) / 2 for s in shape[::-1])  # (x, y, z)
    if cfg == 1:
        return syn.translation((1.3, -0.7, 0.4))
    if cfg == 2:
        return syn.strain_z_plus_sine(0.02, 0.5, 64.0, centre)
    if cfg == 3:
        return syn.rotation_z_hydrostatic(5.0, 0.01, centre)
    if cfg == 5:
        nz, ny, nx = shape
        return syn.indentation(10.5, 80.0, ((nx - 1) / 2, (ny - 1) / 2), 0.3, shape, seed=505)
    raise ValueError(cfg)


def host_pair(cfg: int, seed: int = 1000) -> syn.VolumePair:
    """NumPy-rendered pair for configurations 1-3."""
    shape = shape_of(cfg)
    disp = displacement(cfg)
    if cfg in (1, 2):
        return syn.bead_pair(shape, density=0.02, sigma=1.5, seed=seed + cfg, disp=disp, noise=0.01)
    if cfg == 3:
        pair = syn.bead_pair(shape, density=0.02, sigma=1.5, seed=seed + cfg, disp=disp, noise=0.01, uint16_max=4095)
        nz, ny, nx = shape
        z, y, x = np.ogrid[:nz, :ny, :nx]
        r2 = (x - (nx - 1) / 2) ** 2 + (y - (ny - 1) / 2) ** 2 + (z - (nz - 1) / 2) ** 2
        pair.mask = (r2 <= 110.0**2).astype(np.uint8)
        return pair
    raise ValueError("configuration 5 is rendered on the device: use device_pair(5)")


def host_box(cfg: int, box, seed: int = 1000):
    """(f, g, mask) NumPy volumes of the box ((z0, z1), (y0, y1), (x0, x1)) of a configuration's pair, without the
    device.  Configurations 1 and 2 are cropped from ``host_pair``.  For 3 and 5 the box is rendered from the same
    beads and field as ``device_pair`` (every bead whose support reaches the box), with the same noise model drawn
    on the host (another realisation) and scaled to uint16 over the box."""
    (z0, z1), (y0, y1), (x0, x1) = box
    sl = (slice(z0, z1), slice(y0, y1), slice(x0, x1))
    if cfg in (1, 2):
        pair = host_pair(cfg, seed)
        return np.ascontiguousarray(pair.f[sl]), np.ascontiguousarray(pair.g[sl]), None
    shape = shape_of(cfg)
    disp = displacement(cfg)
    density, sigma, photons = (0.02, 1.5, None) if cfg == 3 else (0.005, 2.0, 1000.0)
    centres, peaks = syn.draw_beads(shape, density, seed + cfg)
    R = int(np.ceil(4.0 * sigma)) + 1
    lo = np.array([z0, y0, x0], dtype=np.float64)
    hi = np.array([z1, y1, x1], dtype=np.float64)
    bshape = (z1 - z0, y1 - y0, x1 - x0)
    vols = []
    for k, c in enumerate((centres, syn.displace_beads(centres, disp))):
        near = np.all((c >= lo - R) & (c < hi + R), axis=1)
        v = syn.render_beads(bshape, c[near] - lo[None, :], peaks[near], sigma).astype(np.float64)
        rng = np.random.default_rng(seed + cfg + 101 + k)
        if photons is not None:
            v = rng.poisson(np.maximum(v, 0.0) * photons) / photons
        vols.append(v + rng.normal(0.0, 0.01, size=v.shape))
    vmin = min(v.min() for v in vols)
    scale = 4095.0 / max(max(v.max() for v in vols) - vmin, 1e-12)
    f, g = (np.round((v - vmin) * scale).astype(np.uint16) for v in vols)
    mask = None
    if cfg == 3:
        nz, ny, nx = shape
        z, y, x = np.ogrid[z0:z1, y0:y1, x0:x1]
        mask = ((x - (nx - 1) / 2) ** 2 + (y - (ny - 1) / 2) ** 2 + (z - (nz - 1) / 2) ** 2 <= ROI_RADIUS**2).astype(np.uint8)
    return f, g, mask


def device_pair(cfg: int, seed: int = 1000, shape=None):
    """(f, g, mask, field): CUDA tensors of the configuration (uint16 for 3 and 5, float32 otherwise).  ``shape``
    renders configuration 3 or 5's beads, noise and field on a volume of another size (profiling cases)."""
    import torch

    from . import kernels as K

    if cfg not in (3, 5):
        if shape is not None:
            raise ValueError("configurations 1 and 2 have their own size")
        pair = host_pair(cfg, seed)
        f = torch.from_numpy(np.ascontiguousarray(pair.f)).cuda()
        g = torch.from_numpy(np.ascontiguousarray(pair.g)).cuda()
        m = None if pair.mask is None else torch.from_numpy(pair.mask).cuda()
        return f, g, m, pair.disp
    # 3: beads 0.02 / voxel, sigma 1.5, Gaussian noise 0.01, spherical ROI; 5: 0.005 / voxel, sigma 2,
    # Poisson (1000 photons per unit peak) plus Gaussian noise 0.01.  Both scaled to uint16 0-4095.
    shape = shape_of(cfg) if shape is None else tuple(int(v) for v in shape)
    disp = displacement(cfg, shape)
    density, sigma, poisson = (0.02, 1.5, False) if cfg == 3 else (0.005, 2.0, True)
    centres, peaks = syn.draw_beads(shape, density, seed + cfg)
    moved = syn.displace_beads(centres, disp)
    R = int(np.ceil(4.0 * sigma))
    vols = []
    for k, c in enumerate((centres, moved)):
        acc = torch.zeros(shape, dtype=torch.float64, device="cuda")
        K.render_beads(acc, c, peaks, sigma, R)
        gen = torch.Generator(device="cuda")
        gen.manual_seed(seed + cfg + 1 + k)
        if poisson:
            photons = 1000.0
            v = torch.poisson(acc.clamp_min(0.0) * photons, generator=gen) / photons
        else:
            v = acc.clone()
        del acc
        v = v + 0.01 * torch.randn(shape, dtype=torch.float64, device="cuda", generator=gen)
        vols.append(v)
    lo = min(float(vols[0].min()), float(vols[1].min()))
    hi = max(float(vols[0].max()), float(vols[1].max()))
    scale = 4095.0 / max(hi - lo, 1e-12)
    out = [torch.round((v - lo) * scale).to(torch.int32).to(torch.uint16).contiguous() for v in vols]
    del vols
    torch.cuda.empty_cache()
    mask = None
    if cfg == 3:
        nz, ny, nx = shape
        z, y, x = (torch.arange(n, device="cuda", dtype=torch.float64) for n in (nz, ny, nx))
        r2 = ((x[None, None, :] - (nx - 1) / 2) ** 2 + (y[None, :, None] - (ny - 1) / 2) ** 2
              + (z[:, None, None] - (nz - 1) / 2) ** 2)
        mask = (r2 <= (ROI_RADIUS * min(shape) / 256.0) ** 2).to(torch.uint8).contiguous()
    return out[0], out[1], mask, disp


def truth_at(disp, coords) -> np.ndarray:
    c = np.asarray(coords, dtype=np.float64)
    return np.column_stack(disp(c[:, 0], c[:, 1], c[:, 2]))
