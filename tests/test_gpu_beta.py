"""GPU: the ADMM penalty auto-tune against the reference's own sweep (tests/golden/golden_beta.npz, made by
tests/golden/make_golden.py from solver/beta_tuning.py:36-109).

Parity bar: candidate betas and the chosen index identical; Err1, Err2 and the scores within 1e-7 relative (each
global step is the PCG to 1e-10 here and a direct sparse solve in the reference).
"""

from __future__ import annotations

import os
from types import SimpleNamespace

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope="module")
def bt():
    with np.load(os.path.join(HERE, "golden", "golden_beta.npz")) as z:
        return {k: z[k] for k in z.files}


@pytest.mark.parametrize("criterion", ["matlab", "normalized"])
def test_auto_tune_beta_matches_reference(bt, criterion):
    from pyaldvc_b200.beta_tuning import auto_tune_beta
    from pyaldvc_b200.subpb2_solver import HexGrid

    grid = HexGrid(tuple(int(g) for g in bt["bt_grid"]), tuple(float(s) for s in bt["bt_spacing"]), bt["bt_elem_active"])
    para = SimpleNamespace(winstepsize=(6, 6, 6), beta_criterion=criterion, alpha=0.0, pcg_tol=1e-10, pcg_max_iter=500)
    beta, info = auto_tune_beta(grid, para, 1e-3, bt["bt_U1"], bt["bt_F1"], bt["bt_exclude"])
    np.testing.assert_allclose(info["betas"], bt[f"bt_{criterion}_betas"], rtol=1e-15)
    np.testing.assert_allclose(info["err1"], bt[f"bt_{criterion}_err1"], rtol=1e-7)
    np.testing.assert_allclose(info["err2"], bt[f"bt_{criterion}_err2"], rtol=1e-7)
    np.testing.assert_allclose(info["score"], bt[f"bt_{criterion}_score"], rtol=1e-6, atol=1e-9)
    assert info["k_best"] == int(bt[f"bt_{criterion}_k_best"])
    assert beta == pytest.approx(float(bt[f"bt_{criterion}_beta"]), rel=1e-9)


def test_pass_with_tuned_beta():
    """A pass with beta=None tunes it over the candidates and runs the ADMM loop with the chosen value."""
    import torch

    from pyaldvc_b200 import configs
    from pyaldvc_b200.beta_tuning import beta_candidates
    from pyaldvc_b200.pipeline import run_pass

    pair = configs.host_pair(2)
    f, g = (torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in (pair.f, pair.g))
    p = configs.params(2, use_global_step=True, beta=None, admm_max_iter=2, autotune=False)
    res = run_pass(f, g, p)
    cands = beta_candidates(p.winstepsize, p.mu, p.beta_range)
    assert res.beta_sweep is not None and res.beta in list(cands)
    assert np.isfinite(res.U.cpu().numpy()).all()
    truth = configs.truth_at(pair.disp, res.coords.cpu().numpy())
    ok = res.valid.cpu().numpy()
    assert np.sqrt(np.mean((res.U.cpu().numpy()[ok] - truth[ok]) ** 2)) < 0.05
