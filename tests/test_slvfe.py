"""slvfe's free-energy functional: product module against the restatement.

ermod_openacc_b200.slvfe (vectorised, the library's downstream step) and
oracle/slvfe_oracle.py (slvfe.F90 restated loop by loop) must agree on
energy distributions produced by the FP64 oracle engine, and both must
satisfy the identities the functional has by construction.
"""
import numpy as np
import pytest

from ermod_openacc_b200 import slvfe as SF
from ermod_openacc_b200 import systems as S
from ermod_openacc_b200 import _capi as A


def synthetic(nbins=120, seed=3):
    rng = np.random.default_rng(seed)
    crd = np.concatenate([np.linspace(-8.0, -0.05, nbins // 2), np.linspace(0.05, 40.0, nbins // 2)])
    rho0 = rng.uniform(0.5, 2.0, nbins)
    rho0 *= 100.0 / rho0.sum()
    chi0 = np.outer(rho0, rho0) + np.diag(rho0)
    return crd, rho0, chi0


def test_identical_distributions_give_aveuv(slvfe_oracle):
    crd, rho0, chi0 = synthetic()
    spec = np.ones(len(crd), dtype=int)
    for f in (SF.delta_mu, slvfe_oracle.delta_mu):
        per, tot = f(rho0, rho0, chi0, crd, spec, 300.0, [-3.25], slfeng=0.5)
        assert per[0] == pytest.approx(-3.25, abs=1e-10)
        assert tot == pytest.approx(-2.75, abs=1e-10)


def test_kT_matches_slvfe():
    assert SF.kT_of(300.0) == pytest.approx(300.0 * 8.314510e-3 / 4.184, rel=1e-15)


def test_product_matches_restatement_on_synthetic_shift(slvfe_oracle):
    crd, rho0, chi0 = synthetic(seed=5)
    spec = np.ones(len(crd), dtype=int)
    rho = rho0 * np.exp(-0.3 * np.tanh(crd / 3.0))
    rho[-5:] = 0.0                      # core bins empty in solution
    rho *= 100.0 / rho.sum()
    a = SF.delta_mu(rho, rho0, chi0, crd, spec, 300.0, [-1.0])
    b = slvfe_oracle.delta_mu(rho, rho0, chi0, crd, spec, 300.0, [-1.0])
    np.testing.assert_allclose(a[0], b[0], rtol=1e-10, atol=1e-10)


def _distributions(oracle_mod):
    """rho from a soln run of an LJ site in water, rho0/chi0 from refs insertions of the same site."""
    w = S.make_workload(1, small=True)
    orc = oracle_mod.Oracle(w.params, w.topo, w.hist, precision=8)
    for fr in range(3):
        pos, cell = w.frame(fr)
        assert orc.engconst(fr + 1, pos, cell) >= 0
    sln = orc.accum(normalise=True)
    topo = S.Topology([S.water(), S.lj_site()], [w.nside ** 3, 1], [A.PT_SOLVENT, A.PT_TEST_RIGID])
    prm = S.default_params(ms1max=32, maxins=3000)
    ref = oracle_mod.Oracle(prm, topo, w.hist, precision=8)
    wr = S.Workload("refs-ljsite", prm, topo, {}, w.box, w.nside, 4, w.seed + 11)
    for fr in range(4):
        pos, cell = wr.frame(fr)
        assert ref.engconst(fr + 1, pos, cell) >= 0
    rfa = ref.accum(normalise=True)
    return orc, sln, rfa


def test_product_matches_restatement_on_engine_distributions(oracle_mod, slvfe_oracle):
    orc, sln, rfa = _distributions(oracle_mod)
    spec = np.ones(orc.ermax, dtype=int)
    aveuv = [float(sln["slnuv"][0])]    # engstore-normalised: aveuv (engproc.F90:622)
    a = SF.delta_mu(sln["edens"], rfa["edens"], rfa["ecorr"], orc.uvcrd, spec, 300.0, aveuv)
    b = slvfe_oracle.delta_mu(sln["edens"], rfa["edens"], rfa["ecorr"], orc.uvcrd, spec, 300.0, aveuv)
    assert np.isfinite(a[1]) and abs(a[1]) < 1e3
    assert a[1] == pytest.approx(b[1], rel=1e-6, abs=1e-6)


@pytest.mark.parametrize("functional,et", [("hnc", 0.0), ("thnc", -0.5), ("thnc", 0.3), ("none", 0.0)])
def test_functionals_match_restatement(slvfe_oracle, functional, et):
    """chmpot's other functionals (slvfe.F90:759-774, thnc :1417-1436) against the loop-by-loop
    restatement on two species."""
    rho, rho0, chi0, crd, spec = _two_species()
    a = SF.delta_mu(rho, rho0, chi0, crd, spec, 300.0, [-1.0, -0.4], functional=functional, et=et)
    b = slvfe_oracle.delta_mu(rho, rho0, chi0, crd, spec, 300.0, [-1.0, -0.4], functional=functional, et=et)
    np.testing.assert_allclose(a[0], b[0], rtol=1e-9, atol=1e-9)


def test_thnc_threshold_limits():
    """thnc with a threshold below every reference-side PMF is hnc; 'none' drops the integrand."""
    rho, rho0, chi0, crd, spec = _two_species()
    hnc = SF.delta_mu(rho, rho0, chi0, crd, spec, 300.0, [-1.0, -0.4], functional="hnc")[1]
    thnc = SF.delta_mu(rho, rho0, chi0, crd, spec, 300.0, [-1.0, -0.4], functional="thnc", et=-1e30)[1]
    assert thnc == pytest.approx(hnc, rel=1e-14)
    with pytest.raises(ValueError):
        SF.delta_mu(rho, rho0, chi0, crd, spec, 300.0, [-1.0, -0.4], functional="pyhnc")


def _ill_conditioned():
    """One species whose chi0 - rho0 rho0^T has a near-null direction besides the constant one:
    the regularised Cholesky solve then returns a huge solution element, which posv_wrap
    (slvfe.F90:520-531) rejects, and getinscv falls back to the eigen-decomposition."""
    crd, rho0, chi0 = synthetic(seed=9)
    n = len(crd)
    v = np.sin(np.arange(n) * 0.37)
    v -= v.mean()
    v /= np.linalg.norm(v)
    A = chi0 - np.outer(rho0, rho0)
    lam, vec = np.linalg.eigh(A)
    A = A - (v @ A @ v - 1e-12) * np.outer(v, v)
    chi = A + np.outer(rho0, rho0)
    rho = rho0 * (1.0 + 0.05 * v * np.sqrt(n))
    rho = np.clip(rho, 1e-3, None)
    rho *= rho0.sum() / rho.sum()
    return rho, rho0, chi, crd, np.ones(n, dtype=int)


def test_posv_rejection_falls_back_to_evd(slvfe_oracle):
    rho, rho0, chi, crd, spec = _ill_conditioned()
    a = SF.delta_mu(rho, rho0, chi, crd, spec, 300.0, [-1.0])
    b = slvfe_oracle.delta_mu(rho, rho0, chi, crd, spec, 300.0, [-1.0])
    assert np.isfinite(a[1]) and abs(a[1]) < 1e3
    np.testing.assert_allclose(a[0], b[0], rtol=1e-7, atol=1e-7)


# ---------------------------------------------------------------------------
# The GPU functional (include/ermod_slvfe.h) against the host module
# ---------------------------------------------------------------------------
def _two_species(seed=7):
    rng = np.random.default_rng(seed)
    crd1, r01, _ = synthetic(80, seed)
    crd2 = np.concatenate([np.linspace(-3.0, -0.02, 20), np.linspace(0.02, 15.0, 40)])
    r02 = rng.uniform(0.5, 2.0, len(crd2))
    r02 *= 30.0 / r02.sum()
    crd = np.concatenate([crd1, crd2])
    rho0 = np.concatenate([r01, r02])
    chi0 = np.outer(rho0, rho0) + np.diag(rho0)
    spec = np.concatenate([np.ones(len(crd1), dtype=int), np.full(len(crd2), 2)])
    rho = rho0 * np.exp(-0.2 * np.tanh(crd / 2.0))
    rho[len(crd1) - 4:len(crd1)] = 0.0
    for p, n in ((1, 100.0), (2, 30.0)):
        rho[spec == p] *= n / rho[spec == p].sum()
    return rho, rho0, chi0, crd, spec


@pytest.mark.gpu
def test_gpu_functional_matches_host_on_synthetic(engine_lib):
    crd, rho0, chi0 = synthetic(seed=5)
    spec = np.ones(len(crd), dtype=int)
    rho = rho0 * np.exp(-0.3 * np.tanh(crd / 3.0))
    rho[-5:] = 0.0
    rho *= 100.0 / rho.sum()
    a = SF.delta_mu(rho, rho0, chi0, crd, spec, 300.0, [-1.0], slfeng=0.25)
    b = SF.delta_mu_gpu(rho, rho0, chi0, crd, spec, 300.0, [-1.0], slfeng=0.25)
    np.testing.assert_allclose(b[0], a[0], rtol=1e-9, atol=1e-9)
    assert b[1] == pytest.approx(a[1], abs=1e-9)
    per, tot = SF.delta_mu_gpu(rho0, rho0, chi0, crd, spec, 300.0, [-3.25], slfeng=0.5)
    assert per[0] == pytest.approx(-3.25, abs=1e-10) and tot == pytest.approx(-2.75, abs=1e-10)


@pytest.mark.gpu
def test_gpu_functional_two_species(engine_lib):
    rho, rho0, chi0, crd, spec = _two_species()
    a = SF.delta_mu(rho, rho0, chi0, crd, spec, 300.0, [-1.0, -0.4])
    b = SF.delta_mu_gpu(rho, rho0, chi0, crd, spec, 300.0, [-1.0, -0.4])
    np.testing.assert_allclose(b[0], a[0], rtol=1e-9, atol=1e-9)


@pytest.mark.gpu
@pytest.mark.parametrize("group,inft", [(1, 0), (3, 0), (5, 80)])
def test_gpu_functional_on_engine_distributions(engine_lib, oracle_mod, group, inft):
    """rho, rho0 and chi0 from the FP64 oracle engine (LJ site in water), bin middles as slvfe
    reads them; group 3 is the bin merging the reference reports (pickgr), (5, 80) one of the
    infchk 'yes' sets."""
    orc, sln, rfa = _distributions(oracle_mod)
    _, middle, _, spec = SF.representative_bins(orc.uvcrd, orc.uvmax, orc.uvsoft)
    aveuv = [float(sln["slnuv"][0])]
    a = SF.delta_mu(sln["edens"], rfa["edens"], rfa["ecorr"], middle, spec, 300.0, aveuv, group=group, inft=inft)
    b = SF.delta_mu_gpu(sln["edens"], rfa["edens"], rfa["ecorr"], middle, spec, 300.0, aveuv, group=group,
                        inft=inft)
    assert np.isfinite(b[1])
    # a 1396-bin regularised solve: FP64 rounding of two Cholesky orders, far below slvfe's 0.01
    assert b[1] == pytest.approx(a[1], abs=1e-6)


@pytest.mark.gpu
def test_gpu_functional_failures(engine_lib):
    crd, rho0, chi0 = synthetic(seed=5)
    spec = np.ones(len(crd), dtype=int)
    with pytest.raises(RuntimeError, match="slv_zer"):        # no bin pair around zero
        SF.delta_mu_gpu(rho0, rho0, chi0, np.abs(crd) + 0.1, spec, 300.0, [0.0])
    with pytest.raises(RuntimeError, match="slv_chl"):        # chi0 - rho0 rho0^T negative definite
        SF.delta_mu_gpu(rho0, rho0, np.outer(rho0, rho0) - 0.5 * np.diag(rho0), crd, spec, 300.0, [0.0],
                        evd=False)
    with pytest.raises(RuntimeError, match="slv_nrm"):        # no correlation at all
        SF.delta_mu_gpu(rho0, rho0, np.zeros_like(chi0), crd, spec, 300.0, [0.0])


@pytest.mark.parametrize("group", [2, 3, 5])
def test_bin_merging_matches_restatement(slvfe_oracle, group):
    """chmpot's grouping (slvfe.F90:609-698): merged arrays and delta mu of the product module
    against the loop-by-loop restatement, two species of uneven bin counts."""
    rho, rho0, chi0, crd, spec = _two_species()
    a = SF.merge_bins(rho, rho0, chi0, crd, spec, group)
    b = slvfe_oracle.merge_bins(rho, rho0, chi0, crd, spec, group)
    for x, y in zip(a, b):
        np.testing.assert_allclose(x, y, rtol=1e-13, atol=1e-13)
    # the last merged bin of a species keeps its last coordinate and takes the remainder
    n1 = int((spec == 1).sum())
    assert a[3][n1 // group - 1] == crd[n1 - 1]
    pa = SF.delta_mu(rho, rho0, chi0, crd, spec, 300.0, [-1.0, -0.4], group=group)
    pb = slvfe_oracle.delta_mu(rho, rho0, chi0, crd, spec, 300.0, [-1.0, -0.4], group=group)
    np.testing.assert_allclose(pa[0], pb[0], rtol=1e-9, atol=1e-9)


def test_identical_distributions_give_aveuv_merged():
    crd, rho0, chi0 = synthetic()
    spec = np.ones(len(crd), dtype=int)
    per, tot = SF.delta_mu(rho0, rho0, chi0, crd, spec, 300.0, [-3.25], slfeng=0.5, group=3)
    assert per[0] == pytest.approx(-3.25, abs=1e-10) and tot == pytest.approx(-2.75, abs=1e-10)


@pytest.mark.gpu
@pytest.mark.parametrize("group", [2, 3])
def test_gpu_functional_merged_bins(engine_lib, group):
    rho, rho0, chi0, crd, spec = _two_species()
    a = SF.delta_mu(rho, rho0, chi0, crd, spec, 300.0, [-1.0, -0.4], group=group)
    b = SF.delta_mu_gpu(rho, rho0, chi0, crd, spec, 300.0, [-1.0, -0.4], group=group)
    np.testing.assert_allclose(b[0], a[0], rtol=1e-9, atol=1e-9)
    with pytest.raises(RuntimeError, match="slv_grp"):
        SF.delta_mu_gpu(rho, rho0, chi0, crd, spec, 300.0, [-1.0, -0.4], group=1000)


@pytest.mark.parametrize("group,inft", [(1, 60), (1, 100), (5, 80), (2, 0)])
def test_core_merging_matches_restatement(oracle_mod, slvfe_oracle, group, inft):
    """inft > 0 (infchk 'yes'): the last rduvcore * inft / 100 core bins of each species join
    its last merged bin; rduvcore counted from the bin coordinates as datread does, on the
    engine's own mesh (linear soft region, logarithmic core)."""
    orc, sln, rfa = _distributions(oracle_mod)
    _, middle, _, spec = SF.representative_bins(orc.uvcrd, orc.uvmax, orc.uvsoft)
    core = SF.core_counts(middle, spec)[1]
    assert core > 50                     # the logarithmic core of the mesh
    a = SF.merge_bins(sln["edens"], rfa["edens"], rfa["ecorr"], middle, spec, group, inft)
    b = slvfe_oracle.merge_bins(sln["edens"], rfa["edens"], rfa["ecorr"], middle, spec, group, inft)
    assert len(a[0]) == (len(middle) - core * inft // 100) // group
    for x, y in zip(a, b):
        np.testing.assert_allclose(x, y, rtol=1e-12, atol=1e-12)


@pytest.mark.gpu
@pytest.mark.parametrize("functional,et", [("hnc", 0.0), ("thnc", 0.3), ("none", 0.0)])
def test_gpu_functionals_match_host(engine_lib, functional, et):
    rho, rho0, chi0, crd, spec = _two_species()
    a = SF.delta_mu_gpu(rho, rho0, chi0, crd, spec, 300.0, [-1.0, -0.4], functional=functional, et=et)
    b = SF.delta_mu(rho, rho0, chi0, crd, spec, 300.0, [-1.0, -0.4], functional=functional, et=et)
    np.testing.assert_allclose(a[0], b[0], rtol=1e-9, atol=1e-9)


@pytest.mark.gpu
def test_gpu_evd_fallback_matches_host(engine_lib):
    """posv_wrap rejects the regularised solution (an element above 1e6); the GPU then solves
    by the eigen-decomposition of the unregularised matrix, as the host module does."""
    rho, rho0, chi, crd, spec = _ill_conditioned()
    info = {}
    a = SF.delta_mu_gpu(rho, rho0, chi, crd, spec, 300.0, [-1.0], info=info)
    assert info["used_evd"]
    b = SF.delta_mu(rho, rho0, chi, crd, spec, 300.0, [-1.0])
    np.testing.assert_allclose(a[0], b[0], rtol=1e-7, atol=1e-7)
    with pytest.raises(RuntimeError, match="slv_chl"):
        SF.delta_mu_gpu(rho, rho0, chi, crd, spec, 300.0, [-1.0], evd=False)
    # a matrix the Cholesky factor rejects outright goes the same way
    crd2, r0, _ = synthetic()
    sp2 = np.ones(len(crd2), dtype=int)
    chi_bad = np.outer(r0, r0) - 0.5 * np.diag(r0)
    info = {}
    r = r0 * np.exp(-0.3 * np.tanh(crd2 / 3.0))
    g = SF.delta_mu_gpu(r, r0, chi_bad, crd2, sp2, 300.0, [0.0], info=info)
    assert info["used_evd"]
    h = SF.delta_mu(r, r0, chi_bad, crd2, sp2, 300.0, [0.0])
    np.testing.assert_allclose(g[0], h[0], rtol=1e-7, atol=1e-7)
