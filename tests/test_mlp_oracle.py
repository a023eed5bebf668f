"""The proposal network's numpy restatement: BF16 rounding and its own gradient."""
import numpy as np
import pytest
import torch

from ermod_openacc_b200 import proposal as P


def test_layout_matches_library_constant(engine_lib):
    import mlp_oracle as M
    assert M.layout()["n"] == P.layout()["n"] == engine_lib.ermod_mlp_nparams() == 41473


def test_bf16_rounding_matches_torch():
    import mlp_oracle as M
    x = np.random.default_rng(0).normal(size=10000).astype(np.float32) * 10.0
    ref = torch.from_numpy(x).to(torch.bfloat16).float().numpy()
    np.testing.assert_array_equal(M.bf16_round(x), ref)


def test_oracle_gradient_by_finite_differences():
    import mlp_oracle as M
    rng = np.random.default_rng(1)
    p = P.init_params(3).astype(np.float64)
    p[P.layout()["b1"][0]:] += rng.normal(0, 0.05, len(p) - P.layout()["b1"][0])
    x = rng.uniform(0, 2, size=(16, 64))
    y = (rng.uniform(size=16) < 0.3).astype(np.float64)
    loss, g = M.loss_and_grad(p, x, y, round_weights=False)
    for idx in rng.choice(len(p), 40, replace=False):
        h = 1e-6
        pp, pm = p.copy(), p.copy()
        pp[idx] += h
        pm[idx] -= h
        fd = (M.loss_and_grad(pp, x, y, False)[0] - M.loss_and_grad(pm, x, y, False)[0]) / (2 * h)
        assert fd == pytest.approx(g[idx], abs=1e-7, rel=1e-4)
