"""The scheduler network's CPU FP64 restatement, checked by central finite
differences (no GPU)."""
import numpy as np

from oracle import mlp_oracle as M


def test_param_count_matches_header():
    from cggraph_b200 import _lib
    assert M.NPARAMS == _lib.POLICY_PARAMS == 6670
    assert M.O == _lib.POLICY_OUTPUTS == 14


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    p = rng.normal(0, 0.2, M.NPARAMS)
    X = rng.random((40, 24))
    T = rng.normal(0, 1, (40, M.O))
    mask = (rng.random((40, M.O)) < 0.5).astype(np.uint8)
    _, g = M.loss_grad(p, X, T, mask)
    idx = rng.choice(M.NPARAMS, 60, replace=False)
    fd = M.finite_diff(p, X, T, mask, idx)
    assert np.max(np.abs(fd - g[idx]) / (np.abs(fd) + 1e-6)) < 1e-4
