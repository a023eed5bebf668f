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


def test_tf32_rounding_is_nearest_ties_away():
    import mlp_oracle as M
    rng = np.random.default_rng(2)
    x = (rng.normal(size=20000) * 10.0 ** rng.uniform(-3, 3, 20000)).astype(np.float32)
    r = M.tf32_round(x).astype(np.float64)
    # 10 explicit mantissa bits: the low 13 bits of the FP32 pattern are zero
    assert np.all((M.tf32_round(x).view(np.uint32) & 0x1FFF) == 0)
    m, e = np.frexp(x.astype(np.float64))           # x = m 2^e, 0.5 <= |m| < 1
    ulp = np.ldexp(1.0, e - 11)                      # TF32 ulp at x's binade
    d = np.abs(r - x)
    assert np.all(d <= 0.5 * ulp)
    ties = d == 0.5 * ulp
    assert np.all(np.abs(r[ties]) > np.abs(x[ties].astype(np.float64)))
    # exact ties, built on purpose: the half-ulp bit set and nothing below it
    u = (np.uint32(0x3F800000) + (np.arange(1, 200, dtype=np.uint32) << 13) + np.uint32(0x1000)).view(np.float32)
    ru = M.tf32_round(u).astype(np.float64)
    assert np.all(ru > u.astype(np.float64))
    assert np.all(M.tf32_round(-u) == -M.tf32_round(u))


def test_gradient_at_given_activations_equals_own_forward():
    import mlp_oracle as M
    rng = np.random.default_rng(3)
    p = P.init_params(5)
    x = rng.uniform(0, 2, size=(32, 64)).astype(np.float32)
    y = (rng.uniform(size=32) < 0.3).astype(np.float64)
    _, (_, h1, h2, h3) = M.forward(p, x, tf32_inputs=True)
    l0, g0 = M.loss_and_grad(p, x, y, tf32_inputs=True)
    l1, g1 = M.loss_and_grad(p, x, y, tf32_inputs=True, acts=(h1, h2, h3))
    assert l1 == pytest.approx(l0, rel=1e-14)
    np.testing.assert_allclose(g1, g0, rtol=1e-12, atol=1e-15)
