"""GPU: the device volume filters (``aldvc_sep_filter``, ``aldvc_mask_fill``) against the oracle and the reference's
own outputs, and the pass with the B-spline interpolant and a deformed-frame mask.

Parity bar: the device filter uses the oracle's operation order (FP64 products and sums, no fused multiply-add),
so device and oracle agree bit for bit on every shape; against the reference's golden outputs the bar of
test_oracle_volume_ops.py applies (bit-identical, short mirrored lines within one float32 step).
"""

from __future__ import annotations

import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope="module")
def vg():
    with np.load(os.path.join(HERE, "golden", "golden_volume_ops.npz")) as z:
        return {k: z[k] for k in z.files}


def _dev(a):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


# (nz, ny, nx): x lines over two tiles, z lines over one tile, single-sample lines, a tiny volume
SHAPES = [(10, 17, 197), (3, 40, 450), (230, 9, 33), (1, 1, 1), (1, 5, 1), (5, 3, 2)]


FILTERS = ["bspline", "gauss0.6", "gauss2.0", "gauss15"]


@pytest.mark.parametrize("shape", SHAPES, ids=lambda s: "x".join(map(str, s)))
@pytest.mark.parametrize("filt", FILTERS)
def test_sep_filter_axes_bit_exact_vs_oracle(oracle_mod, shape, filt):
    from pyaldvc_b200 import kernels as K

    seed = 10 * SHAPES.index(shape) + FILTERS.index(filt)
    v = np.random.default_rng(seed).normal(0.0, 3.0, shape).astype(np.float32)
    if filt == "bspline":
        taps, boundary = oracle_mod.bspline_weights(), 0
    else:
        taps, boundary = oracle_mod.gaussian_weights(float(filt[5:])), 1
    assert np.array_equal(K.bspline_taps(), oracle_mod.bspline_weights())
    for axis in (0, 1, 2):
        got = K.sep_filter(_dev(v), axis, taps, boundary).cpu().numpy()
        np.testing.assert_array_equal(got, oracle_mod.sep_filter(v, axis, taps, boundary), err_msg=f"axis {axis}")


def test_prefilter_and_presmooth_match_reference(vg):
    from pyaldvc_b200 import volume_ops as VO

    np.testing.assert_array_equal(VO.prefilter_bspline(vg["vol"]), vg["bspline"])
    for s in ("0.8", "2.0"):
        np.testing.assert_array_equal(VO.presmooth_volume(vg["vol"], float(s)), vg[f"gauss_{s}"])
    np.testing.assert_array_equal(VO.presmooth_volume(vg["small"], 1.0), vg["small_gauss_1.0"])
    got, ref = VO.prefilter_bspline(vg["small"]), vg["small_bspline"]
    np.testing.assert_allclose(got, ref, rtol=0, atol=2.0**-22 * np.abs(ref).max())
    # the device-tensor fast path returns the same values as the host contract
    np.testing.assert_array_equal(VO.prefilter_bspline(_dev(vg["vol"])).cpu().numpy(), vg["bspline"])


def test_prepare_deformed_masks_with_nan(vg):
    from pyaldvc_b200 import volume_ops as VO

    v = vg["vol"]
    mask = np.ones(v.shape, dtype=bool)
    mask[:, 5:9, 100:130] = False
    out = VO.prepare_deformed(v, "bspline", mask=mask)
    assert np.isnan(out[~mask]).all()
    np.testing.assert_array_equal(out[mask], vg["bspline"][mask])
    out_c = VO.prepare_deformed(v, "cubic", mask=mask)
    assert np.isnan(out_c[~mask]).all()
    np.testing.assert_array_equal(out_c[mask], v[mask])
    np.testing.assert_array_equal(VO.prepare_deformed(v, "linear"), v)
    with pytest.raises(ValueError):
        VO.prepare_deformed(v, "cubic", mask=mask[:, :, :-1])
    with pytest.raises(ValueError):
        VO.prepare_deformed(v, "quintic")


def test_sep_filter_refuses_bad_arguments():
    import torch

    import ctypes

    from pyaldvc_b200 import kernels as K

    v = torch.zeros((4, 4, 4), dtype=torch.float32, device="cuda")
    with pytest.raises(ValueError):
        K.sep_filter(v, 0, np.ones(70), 1)  # more than 63 taps each side
    w = np.ones(3)
    ptr = w.ctypes.data_as(ctypes.c_void_p)
    lib = K.lib()
    assert lib.aldvc_sep_filter(K._p(v), K._p(v), 4, 4, 4, 0, ptr, 2, 1, None) != 0  # in == out
    o = torch.empty_like(v)
    assert lib.aldvc_sep_filter(K._p(v), K._p(o), 4, 4, 4, 3, ptr, 2, 1, None) != 0  # axis
    assert lib.aldvc_sep_filter(K._p(v), K._p(o), 4, 4, 4, 0, ptr, 2, 2, None) != 0  # boundary
    torch.cuda.synchronize()


@pytest.fixture(scope="module")
def config1_device():
    import torch

    from pyaldvc_b200 import configs

    pair = configs.host_pair(1)
    f = torch.from_numpy(np.ascontiguousarray(pair.f)).cuda()
    g = torch.from_numpy(np.ascontiguousarray(pair.g)).cuda()
    return f, g, pair.disp


@pytest.mark.parametrize("interp", ["linear", "cubic", "bspline"])
def test_pass_recovers_the_translation(config1_device, interp):
    """Full pass on the 64^3 translation pair: every interpolant recovers (1.3, -0.7, 0.4) within 0.01 voxel RMS."""
    from pyaldvc_b200 import configs
    from pyaldvc_b200.pipeline import run_pass

    f, g, disp = config1_device
    res = run_pass(f, g, configs.params(1, interp_method=interp, autotune=False))
    coords = res.coords.cpu().numpy()
    U = res.U.cpu().numpy()
    truth = configs.truth_at(disp, coords)
    ok = res.status.cpu().numpy() == 0
    assert ok.mean() > 0.9
    rms = float(np.sqrt(np.mean((U[ok] - truth[ok]) ** 2)))
    assert rms < 0.01, f"{interp}: rms {rms:.4f}"


def test_pass_with_deformed_mask(config1_device):
    """An all-material deformed-frame mask changes nothing; a masked slab changes only the nodes whose deformed
    subsets (half-width 10, plus the 2-voxel interpolation stencil) reach it."""
    import torch

    from pyaldvc_b200 import configs
    from pyaldvc_b200.pipeline import run_pass

    f, g, _ = config1_device
    p = configs.params(1, autotune=False)
    base = run_pass(f, g, p)
    ones = run_pass(f, g, p, g_mask=torch.ones(g.shape, dtype=torch.bool, device="cuda"))
    torch.testing.assert_close(ones.U, base.U, rtol=0, atol=0)
    gm = torch.ones(g.shape, dtype=torch.bool, device="cuda")
    gm[:, :, 56:] = False
    slab = run_pass(f, g, p, g_mask=gm)
    x = base.coords[:, 0].cpu().numpy()
    far = x + 10 + 1.3 + 3 < 56
    assert far.any() and (~far).any()
    np.testing.assert_array_equal(slab.U.cpu().numpy()[far], base.U.cpu().numpy()[far])
    assert np.isfinite(slab.U.cpu().numpy()).all()


class _Voi:
    """Inclusive (lo, hi) index ranges with the reference VOIRange's clamp / slices (core/data_structures.py:87-130)."""

    def __init__(self, x, y, z):
        self.x, self.y, self.z = x, y, z

    def clamp(self, shape):
        nz, ny, nx = shape

        def one(r, n):
            lo, hi = int(r[0]), int(r[1])
            hi = n - 1 if hi < 0 else hi
            lo = max(0, min(lo, n - 1))
            return lo, max(lo, min(hi, n - 1))

        return _Voi(one(self.x, nx), one(self.y, ny), one(self.z, nz))

    @property
    def slices(self):
        return slice(self.z[0], self.z[1] + 1), slice(self.y[0], self.y[1] + 1), slice(self.x[0], self.x[1] + 1)


def test_normalize_volume_whole_and_voi_match_reference(vg):
    """normalize_volume (io/volume_ops.py:105-121) of a uint16 volume, whole and over a VOI box: within one float32
    step of the reference (FP64 statistics on both sides, summed in another order), almost all bit-identical."""
    from pyaldvc_b200 import volume_ops as VO

    raw = vg["norm_raw"]
    for got, ref in ((VO.normalize_volume(raw), vg["norm_whole"]),
                     (VO.normalize_volume(raw, _Voi((8, 33), (4, 16), (2, 10))), vg["norm_voi"])):
        np.testing.assert_allclose(got, ref, rtol=0, atol=np.spacing(np.abs(ref).max()))
        assert np.mean(got == ref) > 0.999
    assert not np.allclose(vg["norm_whole"], vg["norm_voi"])  # the VOI statistics differ from the whole volume's
