"""GPU: whole AL-DVC passes on the device (pyaldvc_b200.pipeline.run_pass) against the reference.

- The reference's own run_aldvc (core/pipeline.py:255-366: initial guess, local 12-DOF with outlier filling,
  global step, ADMM with its early stop) on the four seeded pairs of tests/golden/golden_pass.npz.
- The FP64 oracle pass (oracle.aldvc_pass, pinned bit for bit to those fixtures by tests/test_oracle_pass.py)
  on sub-volumes of the benchmark configurations, in the forms the benchmark runs: configuration 2 (25^3
  tricubic subsets, direct NCC +-8), configuration 3 (uint16, spherical mask, uneven 17..33-voxel subsets,
  ADMM captured as a CUDA graph) and configuration 5 (uint16 Poisson beads, 33^3 tricubic subsets on the lean
  4-warp kernel with the overlapping-quad copy, a 17^3 template at +-16 on the in-register FFT engine).
- CUDA-graph replay of the ADMM loop against eager execution, on two different inputs.

Parity bar: displacements within 1e-3 voxel, displacement gradients within 1e-5, identical
node validity and ADMM step counts, identical final statuses.
"""

from __future__ import annotations

import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))

import pass_inputs as PI  # noqa: E402

pytestmark = pytest.mark.gpu

U_TOL = 1e-3  # voxel
F_TOL = 1e-5


@pytest.fixture(scope="module")
def gp():
    with np.load(os.path.join(HERE, "golden", "golden_pass.npz")) as z:
        return {k: z[k] for k in z.files}


def _cuda(a):
    import torch

    return None if a is None else torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _np(t):
    return t.detach().cpu().numpy()


def _check_pass(res, ref: dict, what: str, steps: int | None = None):
    """res: a PassResult; ref: dict with valid, U0, U_local, F_local, U, F, status, admm_steps (numpy)."""
    valid = _np(res.valid)
    np.testing.assert_array_equal(valid, ref["valid"], err_msg=f"{what}: node validity")
    if steps is not None:
        assert res.admm_steps == steps, f"{what}: {res.admm_steps} ADMM steps, reference {steps}"
    N = valid.shape[0]
    for k, got, tol in (("U0", res.U0, U_TOL), ("U_local", res.U_local, U_TOL), ("F_local", res.F_local, F_TOL),
                        ("U", res.U, U_TOL), ("F", res.F, F_TOL)):
        g_ = _np(got).reshape(N, -1)
        r_ = np.asarray(ref[k]).reshape(N, -1)
        d = np.abs(g_ - r_)
        worst = float(np.nanmax(d)) if d.size else 0.0
        assert np.array_equal(np.isnan(g_), np.isnan(r_)), f"{what} {k}: NaN pattern differs"
        assert worst <= tol, f"{what} {k}: max |diff| {worst:.3e} > {tol:g} (rms {float(np.sqrt(np.nanmean(d * d))):.3e})"
    for k, got in (("status_local", res.status_local), ("status", res.status)):
        g_ = _np(got).astype(np.int64)
        r_ = np.asarray(ref[k]).astype(np.int64)
        np.testing.assert_array_equal(g_, r_, err_msg=f"{what} {k}: statuses differ at {np.flatnonzero(g_ != r_)[:10]}")


def _params(name, **over):
    from pyaldvc_b200.pipeline import PassParams

    c = PI.PASS_CASES[name]["para"]
    p = PassParams(winsize=c["winsize"], winstepsize=c["winstepsize"], search_radius=c["search_radius"],
                   interp_method=c["interp_method"], admm_max_iter=c["admm_max_iter"], admm_tol=c.get("admm_tol", 1e-2),
                   init_guess_method="ncc", global_shift=False, beta=PI.PASS_COMMON["beta"], mu=PI.PASS_COMMON["mu"])
    for k, v in over.items():
        setattr(p, k, v)
    return p


@pytest.mark.parametrize("name", list(PI.PASS_CASES))
def test_pass_matches_reference_run_aldvc(gp, name):
    """run_pass on the raw pair (normalisation on the device) against the reference's run_aldvc."""
    from pyaldvc_b200.pipeline import run_pass

    f, g, mask, _ = PI.pass_pair(name)
    res = run_pass(_cuda(f), _cuda(g), _params(name), _cuda(None if mask is None else mask.astype(np.uint8)))
    np.testing.assert_array_equal(_np(res.coords), gp[f"{name}_coords"])
    ref = {"valid": gp[f"{name}_node_valid"], "U0": gp[f"{name}_U0"], "U_local": gp[f"{name}_U_local"],
           "F_local": gp[f"{name}_F_local"], "U": gp[f"{name}_U"], "F": gp[f"{name}_F"], "status": gp[f"{name}_status"],
           "status_local": gp[f"{name}_status_local"]}
    _check_pass(res, ref, f"pass {name}", int(gp[f"{name}_steps"]))


# --------------------------------------------------------------------------- sub-volumes of the benchmark configurations
def _crop_config2():
    """A 64^3 box of configuration 2's pair (2 % z strain + sine), its own node grid: 216 nodes."""
    from pyaldvc_b200 import configs

    pair = configs.host_pair(2)
    sl = (slice(20, 84), slice(30, 94), slice(40, 104))
    p = configs.params(2, autotune=False, threads=128)
    return np.ascontiguousarray(pair.f[sl]), np.ascontiguousarray(pair.g[sl]), None, p, None


def _crop_config3(origin=(100, 60, 40)):
    """A 96^3 box of configuration 3's uint16 pair across the spherical ROI's boundary, with the per-node subset
    shapes of the full volume's rule (16x16x24 at the ROI centre to 32^3 at its edge) and the ROI mask."""
    from pyaldvc_b200 import configs

    pair = _config3_pair()
    z0, y0, x0 = origin
    sl = (slice(z0, z0 + 96), slice(y0, y0 + 96), slice(x0, x0 + 96))
    off = np.array([x0, y0, z0], dtype=np.int64)
    p = configs.params(3, node_winsize=lambda c: configs.uneven_winsize(np.asarray(c) + off[None, :]), threads=128)
    return (np.ascontiguousarray(pair.f[sl]), np.ascontiguousarray(pair.g[sl]), np.ascontiguousarray(pair.mask[sl]), p,
            lambda c: configs.uneven_winsize(np.asarray(c) + off[None, :]) // 2)


_C3 = {}


def _config3_pair():
    from pyaldvc_b200 import configs

    if "pair" not in _C3:
        _C3["pair"] = configs.host_pair(3)
    return _C3["pair"]


def _crop_config5():
    """A 100 x 128 x 128 box at the indenter of configuration 5 (uint16, 0.005 beads / voxel, sigma 2, Poisson plus
    Gaussian noise, Boussinesq field with its background): 320 nodes of 33^3 subsets, NCC +-16 (FFT engine)."""
    from pyaldvc_b200 import configs
    from pyaldvc_b200 import synthetic as syn

    full = configs.displacement(5)
    ox, oy, oz = 448.0, 448.0, 0.0

    def disp(x, y, z):
        return full(x + ox, y + oy, z + oz)

    pair = syn.bead_pair((100, 128, 128), density=0.005, sigma=2.0, seed=505, disp=disp, noise=0.01, poisson_photons=1000.0,
                         uint16_max=4095)
    p = configs.params(5, autotune=False, threads=128)
    return pair.f, pair.g, None, p, None


def _crop_config5_staged():
    """The configuration-5 box with the IC-GN sweeps staged through TMA copies of g."""
    f, g, mask, p, half_of = _crop_config5()
    p.threads, p.brick_floats = 128, -1
    return f, g, mask, p, half_of


CROPS = {"config2": _crop_config2, "config3": _crop_config3, "config5": _crop_config5, "config5_staged": _crop_config5_staged}


def _oracle_pass(oracle_mod, f, g, mask, p, res, half_of):
    """The FP64 oracle pass on the same (host-normalised) volumes, grid and parameters."""
    fn, gn = oracle_mod.normalize_volume(f), oracle_mod.normalize_volume(g)
    coords = _np(res.coords)
    node_half = None if half_of is None else half_of(coords)
    spacing = tuple(float(s) for s in p.winstepsize)
    prm = dict(winsize=p.winsize, search_radius=p.search_radius, interp_method=p.interp_method, mu=p.mu, beta=p.beta,
               admm_max_iter=p.admm_max_iter, admm_tol=p.admm_tol if p.admm_early_stop else -1.0,
               use_global_step=p.use_global_step)
    return oracle_mod.aldvc_pass(fn, gn, coords, res.grid_shape, spacing, mask=None if mask is None else mask != 0,
                                 node_half=node_half, **prm)


@pytest.mark.parametrize("crop", list(CROPS))
def test_pass_on_configuration_subvolume_matches_oracle(oracle_mod, crop):
    from pyaldvc_b200.pipeline import clear_graphs, run_pass

    f, g, mask, p, half_of = CROPS[crop]()
    res = run_pass(_cuda(f), _cuda(g), p, _cuda(mask))
    o = _oracle_pass(oracle_mod, f, g, mask, p, res, half_of)
    clear_graphs()
    ref = {k: o[k] for k in ("valid", "U0", "U_local", "F_local", "U", "F", "status", "status_local")}
    _check_pass(res, ref, crop, o["admm_steps"] if p.use_global_step else None)
    assert np.mean(_np(res.status) == 0) > 0.6, f"{crop}: too few converged nodes to mean anything"


def test_admm_graph_replay_matches_eager():
    """The ADMM loop of the configuration-3 form captured once and replayed on a second input equals eager
    execution of both inputs bit for bit (static inputs refreshed, no stale tensor or cache key)."""
    import torch

    from pyaldvc_b200.pipeline import clear_graphs, graph_count, run_pass

    clear_graphs()
    runs = {}
    for origin in ((100, 60, 40), (60, 100, 120)):
        f, g, mask, p, _ = _crop_config3(origin)
        fd, gd, md = _cuda(f), _cuda(g), _cuda(mask)
        p.graph = True
        r_graph = run_pass(fd, gd, p, md)
        n_graphs = graph_count()
        p.graph = False
        r_eager = run_pass(fd, gd, p, md)
        runs[origin] = (r_graph, r_eager, n_graphs)
    clear_graphs()
    (a_g, a_e, n1), (b_g, b_e, n2) = runs.values()
    assert n1 == 1 and n2 == 1, "the second input must replay the graph captured by the first"
    for r_g, r_e in ((a_g, a_e), (b_g, b_e)):
        assert r_g.admm_steps == r_e.admm_steps
        for k in ("U", "F", "status", "zncc", "n_iter"):
            x, y = getattr(r_g, k), getattr(r_e, k)
            same = (x == y) | (torch.isnan(x) & torch.isnan(y)) if x.is_floating_point() else x == y  # NaN at rejected nodes
            assert bool(same.all()), f"graph replay differs from eager in {k}"
    assert not torch.equal(a_g.U, b_g.U)


def test_pass_from_host_buffers_equals_device_inputs():
    """Host inputs (pinned and pageable) are copied within the pass, the reference frame first and the deformed
    frame behind its preparation: the pass equals the one on device inputs bit for bit (configuration-3 box: uint16
    pair with its ROI mask), with a prepared reference too (then only the deformed frame is copied)."""
    import torch

    from pyaldvc_b200.pipeline import prepare_reference, run_pass

    f, g, mask, p, _ = _crop_config3()
    dev = run_pass(_cuda(f), _cuda(g), p, _cuda(mask))
    fh, gh, mh = (torch.from_numpy(np.ascontiguousarray(a)) for a in (f, g, mask))
    ref = prepare_reference(_cuda(f), p, _cuda(mask))
    for what, res in (("pinned", run_pass(fh.pin_memory(), gh.pin_memory(), p, mh.pin_memory())),
                      ("pageable", run_pass(fh, gh, p, mh)),
                      ("prepared reference", run_pass(None, gh.pin_memory(), p, ref=ref))):
        assert res.admm_steps == dev.admm_steps, what
        for k in ("U", "F", "U_local", "U0", "status", "zncc"):
            x, y = getattr(res, k), getattr(dev, k)
            same = (x == y) | (torch.isnan(x) & torch.isnan(y)) if x.is_floating_point() else x == y
            assert bool(same.all()), f"{what}: {k} differs from the pass on device inputs"
