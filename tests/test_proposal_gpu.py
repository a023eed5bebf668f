"""The learned insertion proposal on the GPU.

1. The hand-written forward/backward kernels against the numpy restatement
   (oracle/mlp_oracle.py): logits, loss and every parameter gradient.
2. Training on the device lowers the loss.
3. What the trained network gains: on held-out frames, learned insertion
   puts more insertions where the solute fits and estimates the
   uniform-insertion quantity P(E_total < threshold) without bias (p/q
   weights) and with a smaller variance than uniform insertion of the same
   size.
"""
import numpy as np
import pytest

from ermod_openacc_b200 import Engine
from ermod_openacc_b200 import _capi as A
from ermod_openacc_b200 import proposal as P
from ermod_openacc_b200 import systems as S

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lib(engine_lib):
    return engine_lib


def perturbed_params(seed):
    rng = np.random.default_rng(seed)
    p = P.init_params(seed)
    L = P.layout()
    for k in ("b1", "b2", "b3", "b4"):
        off, n = L[k]
        p[off:off + n] = rng.normal(0.0, 0.1, n)
    return p


def test_mlp_forward_and_gradients_match_oracle(lib):
    import mlp_oracle as M
    rng = np.random.default_rng(11)
    p = perturbed_params(4)
    x = rng.uniform(0.0, 3.0, size=(300, 64)).astype(np.float32)
    y = (rng.uniform(size=300) < 0.3).astype(np.float32)
    tr = P.Trainer(p, max_batch=512)
    s_gpu = tr.forward(x)
    s_orc, _ = M.forward(p, x)
    np.testing.assert_allclose(s_gpu, s_orc, rtol=1e-4, atol=1e-4 * np.abs(s_orc).max())
    g_gpu, l_gpu = tr.gradients(x, y)
    l_orc, g_orc = M.loss_and_grad(p, x, y)
    assert l_gpu == pytest.approx(l_orc, rel=1e-5)
    L = P.layout()
    for k in ("W1", "b1", "W2", "b2", "W3", "b3", "w4", "b4"):
        off, n = L[k]
        a, b = g_gpu[off:off + n], g_orc[off:off + n]
        assert np.max(np.abs(a - b)) <= 2e-4 * np.max(np.abs(b)) + 1e-7, k
    tr.close()


def test_training_reduces_loss(lib):
    rng = np.random.default_rng(2)
    x = rng.uniform(0.0, 2.0, size=(8192, 64)).astype(np.float32)
    y = ((x[:, 21] + x[:, 42]) < 1.6).astype(np.float32)
    tr = P.Trainer(P.init_params(1), max_batch=1024)
    hist = tr.fit(x, y, epochs=8, batch=512, lr=2e-3)
    assert hist[-1] < 0.5 * hist[0]
    logits = tr.forward(x[:1024])
    acc = np.mean((logits > 0) == (y[:1024] > 0.5))
    assert acc > 0.9
    tr.close()


def small_refs(nsite, maxins, proposal):
    base = S.make_workload(2, small=True)
    topo = S.Topology([S.water(), S.ring_recipe_solute(nsite, 5)], [base.nside ** 3, 1],
                      [A.PT_SOLVENT, A.PT_TEST_RIGID])
    prm = dict(base.params, maxins=maxins, proposal=proposal, corrcal=0)
    # disordered water: the lattice has no cavities for a voxel proposal to find
    return S.Workload("refs-proposal", prm, topo, {}, base.box, base.nside, 40, base.seed, packing="random"), prm


def test_learned_proposal_is_unbiased_and_gains(lib):
    """Train on uniform insertions of an LJ site in disordered water (labels: the lowest 5% of the
    insertion energies), then compare 8 repeats of learned and uniform insertion on held-out frames:
    the p/q-weighted estimates agree with uniform insertion, more insertions land where the site fits,
    and the excess chemical potential by test-particle insertion, -kT ln <exp(-E/kT)>, which the
    lowest energies dominate, scatters less."""
    gv, eps, nins, kT = 16, 0.2, 2048, 300.0 * S.KB_KCAL
    w, prm = small_refs(1, nins, A.PROPOSAL_UNIFORM)
    eng = Engine(prm, w.topo, w.hist)
    eng.proposal_config(gv, eps, feature_cells=gv)
    feats, etot, _ = P.collect_uniform_samples(eng, [w.frame(i) for i in range(12)])
    y, thr = P.labels_from_energies(etot, quantile=0.05)
    tr = P.Trainer(P.init_params(7), max_batch=2048)
    hist = tr.fit(feats, y, epochs=20, batch=512, lr=1e-3)
    assert hist[-1] < hist[0]
    params = tr.params()
    tr.close()
    eng.close()
    frames = [w.frame(20 + i) for i in range(3)]
    res = {}
    wmean = []
    for mode in (A.PROPOSAL_UNIFORM, A.PROPOSAL_LEARNED):
        widom, frac, hits = [], [], []
        for rep in range(8):
            e = Engine(dict(prm, proposal=mode, iseed=1000 + rep), w.topo, w.hist)
            e.proposal_config(gv, eps, params if mode == A.PROPOSAL_LEARNED else None, feature_cells=gv)
            num = den = fnum = 0.0
            low = 0
            for i, (pos, cell) in enumerate(frames):
                assert e.engconst(i + 1, pos, cell) >= 0
                _, en, _ = e.insertion_samples()
                _, wt = e.insertions()
                num += np.sum(wt * np.exp(-np.minimum(en, 1e4) / kT))
                fnum += np.sum(wt * (en < thr))
                den += np.sum(wt)
                low += np.sum(en < thr)
                if mode == A.PROPOSAL_LEARNED:
                    wmean.append(wt.mean())
            widom.append(-kT * np.log(num / den))
            frac.append(fnum / den)
            hits.append(low / (len(frames) * nins))
            e.close()
        res[mode] = (np.array(widom), np.array(frac), np.mean(hits))
    (wu, fu, hu), (wl, fl, hl) = res[A.PROPOSAL_UNIFORM], res[A.PROPOSAL_LEARNED]
    se = lambda a, b: np.sqrt(a.var(ddof=1) / len(a) + b.var(ddof=1) / len(b))
    assert abs(fu.mean() - fl.mean()) <= 4.0 * se(fu, fl) + 1e-3     # unbiased through p/q
    assert abs(wu.mean() - wl.mean()) <= 4.0 * se(wu, wl)
    assert abs(np.mean(wmean) - 1.0) < 0.1                           # E_q[p/q] = 1
    assert hl > 1.5 * hu                                              # insertions go where the site fits
    assert wl.var(ddof=1) < 0.6 * wu.var(ddof=1)                      # the gain
