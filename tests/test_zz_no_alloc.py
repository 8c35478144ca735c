"""The no-allocation PCG entry point against the workspace one, through the C ABI.

``aldvc_pcg_hex8_noalloc`` serves callers that cannot allocate device memory (a plugin inside a host
application that owns the device budget, a real-time loop that must not call cudaMalloc); its scratch is a
built-in device array shared by every call.  Two calls in a row, each compared with ``aldvc_pcg_hex8`` on
the same inputs: same iteration count, X within 1e-12 (the same kernel in the same order, so in practice
bit-identical), and the second call is not disturbed by the first call's leftovers in the shared array.
This file is collected last so that a run stopping at the first failure has run every other test.
"""

from __future__ import annotations

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _problem(seed: int, grid_shape=(14, 17, 19), spacing=(6.0, 7.0, 5.0)):
    import torch

    rng = np.random.default_rng(seed)
    nz, ny, nx = grid_shape
    n = nz * ny * nx
    elem = (rng.random((nz - 1) * (ny - 1) * (nx - 1)) > 0.1).astype(np.uint8)  # about 10 % of the elements dropped
    B = rng.normal(0.0, 1.0, (n, 3))
    X0 = rng.normal(0.0, 0.3, (n, 3))
    cuda = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    return grid_shape, spacing, cuda(elem), cuda(B), cuda(X0)


def _solve(lib, K, grid_shape, spacing, elem, B, X0, noalloc: bool):
    import torch

    m = K.mesh_struct(grid_shape, spacing, elem, 2)
    X = torch.full_like(B, float("nan"))
    iters = torch.zeros(1, dtype=torch.int32, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    beta, mu, alpha, tol, max_iter = 1e-3, 1e-3, 0.0, 1e-10, 500
    p = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731
    stream = torch.cuda.current_stream().cuda_stream
    if noalloc:
        rc = lib.aldvc_pcg_hex8_noalloc(ctypes.byref(m), beta, mu, alpha, p(B), p(X0), tol, max_iter, p(X), p(iters), p(err),
                                        stream)
    else:
        ws = torch.empty(lib.aldvc_pcg_workspace_size(ctypes.byref(m)), dtype=torch.uint8, device="cuda")
        rc = lib.aldvc_pcg_hex8(ctypes.byref(m), beta, mu, alpha, p(B), p(X0), tol, max_iter, p(ws), ws.numel(), p(X), p(iters),
                                p(err), stream)
    assert rc == 0, lib.aldvc_last_error()
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    return X.cpu().numpy(), int(iters.item())


def test_noalloc_pcg_matches_workspace_pcg_on_two_calls():
    from pyaldvc_b200 import _lib
    from pyaldvc_b200 import kernels as K

    lib = _lib.load()
    for seed in (3, 4):  # two calls in a row through the shared built-in scratch
        prob = _problem(seed)
        X_ref, it_ref = _solve(lib, K, *prob, noalloc=False)
        X_na, it_na = _solve(lib, K, *prob, noalloc=True)
        assert it_na == it_ref and it_ref > 5
        assert np.all(np.isfinite(X_na))
        np.testing.assert_allclose(X_na, X_ref, rtol=0, atol=1e-12)


def test_noalloc_pcg_rejects_meshes_beyond_its_scratch():
    import torch

    from pyaldvc_b200 import _lib
    from pyaldvc_b200 import kernels as K

    lib = _lib.load()
    cap = int(lib.aldvc_pcg_hex8_noalloc_max_nodes())
    assert cap >= 147928  # the 1024 x 1024 x 306 configuration's mesh fits
    m = K.mesh_struct((64, 64, 65), (1.0, 1.0, 1.0), None, 2)  # 266,240 nodes > cap
    dummy = torch.zeros(3, dtype=torch.float64, device="cuda")
    it = torch.zeros(1, dtype=torch.int32, device="cuda")
    p = ctypes.c_void_p(dummy.data_ptr())
    pi = ctypes.c_void_p(it.data_ptr())
    rc = lib.aldvc_pcg_hex8_noalloc(ctypes.byref(m), 1e-3, 1e-3, 0.0, p, p, 1e-8, 10, p, pi, pi, 0)
    assert rc == -1 and b"limit" in lib.aldvc_last_error()
