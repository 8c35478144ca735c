"""GPU: the bounded grid-barrier waits of the cooperative kernels give up, report it and leave the context usable.

The PCG and the inpainting are single cooperative launches whose blocks meet at grid barriers.  A barrier
waits at most a fixed number of polls; a block that runs out sets the launch's error word and returns.  The
test hook aldvc_test_set_barrier makes every barrier wait for one block more than the launch has, so no
barrier ever opens and every wait runs out (a flag that nothing sets), with a spin limit of a fraction of a
millisecond.  The tests check that the kernels return promptly, that the error word is set, that every host
path reports it (the NumPy contract raises, a whole pass raises DeviceError after its single end-of-pass read)
and that the same calls succeed again once the hook is reset.  No GPU fault or hang is involved.
"""

from __future__ import annotations

import os
import sys
import time

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))

pytestmark = pytest.mark.gpu

SPINS = 4096  # polls of about 64 ns before a block gives up


@pytest.fixture()
def give_up():
    from pyaldvc_b200 import kernels as K

    K.test_set_barrier(1, SPINS)
    try:
        yield K
    finally:
        K.test_set_barrier(0, 0)


def _system(golden):
    from pyaldvc_b200.subpb2_solver import HexGrid, build_global_system

    grid = HexGrid(tuple(int(s) for s in golden["pcg_grid_shape"]), tuple(float(s) for s in golden["pcg_spacing"]),
                   golden["pcg_elem_active"])
    return build_global_system(grid, 1e-3, 1e-3, 0.0, pcg_tol=1e-10)


def test_pcg_barrier_gives_up_and_is_reported(golden, give_up):
    import torch

    from pyaldvc_b200.subpb2_solver import solve_subpb2, solve_subpb2_device

    K = give_up
    system = _system(golden)
    args = (golden["pcg_U1"], golden["pcg_F1"], golden["pcg_W"], golden["pcg_v"])
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    _, _, err = solve_subpb2_device(system, *args)
    torch.cuda.synchronize()
    assert time.perf_counter() - t0 < 5.0
    assert int(err.item()) == 1
    with pytest.raises(K.DeviceError):
        solve_subpb2(system, *args)
    K.test_set_barrier(0, 0)  # the context is usable: the same solve now converges to the reference's result
    U2, info = solve_subpb2(system, *args)
    np.testing.assert_allclose(U2, golden["pcg_U2"], rtol=0, atol=1e-8)


def test_noalloc_pcg_barrier_gives_up(golden, give_up):
    """The PCG entry point with built-in scratch gives up the same way (through the C ABI)."""
    import ctypes

    import torch

    K = give_up
    system = _system(golden)
    g = system.grid
    cuda = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    U1 = cuda(golden["pcg_U1"])
    b = K.global_rhs(g.grid_shape, g.spacing, system.elem_device(), 1e-3, 1e-3, 0.0, U1, cuda(golden["pcg_F1"]),
                     cuda(golden["pcg_W"]), cuda(golden["pcg_v"]), g.gauss_order)
    m = K.mesh_struct(g.grid_shape, g.spacing, system.elem_device(), g.gauss_order)
    X = torch.empty_like(U1)
    iters = torch.zeros(1, dtype=torch.int32, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    p = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731
    rc = K.lib().aldvc_pcg_hex8_noalloc(ctypes.byref(m), 1e-3, 1e-3, 0.0, p(b), p(U1), 1e-10, 500, p(X), p(iters), p(err),
                                        torch.cuda.current_stream().cuda_stream)
    assert rc == 0
    assert int(err.item()) == 1


def test_inpainting_barrier_gives_up_and_is_reported(give_up):
    import torch

    K = give_up
    grid = (6, 7, 8)
    rng = np.random.default_rng(3)
    v = torch.from_numpy(rng.normal(size=(int(np.prod(grid)), 3))).cuda()
    unk = torch.from_numpy((rng.random(int(np.prod(grid))) < 0.3).astype(np.uint8)).cuda()
    _, err = K.inpaint(v, grid, unk)
    assert int(err.item()) == 1
    words = K.ErrorWords()
    words.add(err, "inpaint")
    with pytest.raises(K.DeviceError, match="inpaint"):
        words.check()
    _, err = K.median_test(v, grid, (unk == 0).to(torch.uint8), 2.0)  # the median test inpaints its holes first
    assert int(err.item()) == 1


def test_pass_raises_when_a_wait_gives_up(give_up):
    """A whole pass reads its error words once, at the end, and raises; the next pass without the hook succeeds."""
    import torch

    import pass_inputs as PI
    from pyaldvc_b200.pipeline import PassParams, run_pass

    K = give_up
    f, g, _, _ = PI.pass_pair("affine")
    c = PI.PASS_CASES["affine"]["para"]
    p = PassParams(winsize=c["winsize"], winstepsize=c["winstepsize"], search_radius=c["search_radius"], admm_max_iter=2,
                   init_guess_method="ncc", global_shift=False, beta=1e-3, mu=1e-3, autotune=False)
    fd, gd = torch.from_numpy(f).cuda(), torch.from_numpy(g).cuda()
    with pytest.raises(K.DeviceError):
        run_pass(fd, gd, p)
    K.test_set_barrier(0, 0)
    res = run_pass(fd, gd, p)
    assert bool(torch.isfinite(res.U).all())
