"""Pins of the CPU oracle against published known answers (CPU only).

The reference ships no tests or golden vectors and cannot be built here
(Fortran + OpenACC, no Fortran compiler), so the oracle is pinned by:
  * Random123's published Philox4x32-10 known-answer vectors,
  * exact cardinal B-spline values M_4, M_6 (spline.F90:25-58),
  * the reference's own mesh sizes (1396 / 2596 bins for the gen_input /
    parameters_er.example &hist sets, engproc.F90:171-281),
  * binsearch semantics read from engproc.F90:1078-1108,
  * the NaCl Madelung constant and the simple-cubic Wigner constant through
    the full realcal + recpcal + residual chain,
  * analytic LJ pair energies and numpy's FFT for the PME self energy.
"""
import numpy as np
import pytest

from ermod_openacc_b200 import _capi as A
from ermod_openacc_b200 import systems as S
from _helpers import COULOMB, MADELUNG_NACL, WIGNER_SC, nacl_system


def test_philox_known_answers(oracle_mod):
    # Random123 kat_vectors, philox4x32_10
    assert oracle_mod.philox([0, 0, 0, 0], [0, 0]) == [0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8]
    assert oracle_mod.philox([0xffffffff] * 4, [0xffffffff] * 2) == [0x408f276d, 0x41c83b0e, 0xa20bc7c6,
                                                                       0x6d5451fd]
    assert oracle_mod.philox([0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344], [0xa4093822, 0x299f31d0]) == [
        0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1]


@pytest.mark.parametrize("order,x,val", [(4, 1.0, 1 / 6), (4, 2.0, 2 / 3), (4, 3.0, 1 / 6), (4, 0.5, 1 / 48),
                                         (6, 1.0, 1 / 120), (6, 2.0, 26 / 120), (6, 3.0, 66 / 120),
                                         (4, 0.0, 0.0), (4, 4.0, 0.0)])
def test_bspline_values(oracle_mod, order, x, val):
    assert oracle_mod.spline_value(order, x) == pytest.approx(val, rel=1e-14, abs=1e-15)


def test_bspline_partition_of_unity(oracle_mod):
    for order in (4, 6, 8):
        for f in np.linspace(0.0, 0.999, 7):
            s = sum(oracle_mod.spline_value(order, f + k) for k in range(order))
            assert s == pytest.approx(1.0, abs=1e-12)


@pytest.mark.parametrize("ecdmin,ermax,esmax", [(-20.0, 1396, 1196), (-80.0, 2596, 2396)])
def test_mesh_sizes(oracle_mod, ecdmin, ermax, esmax):
    uvcrd, uvmax, uvsoft, escrd = oracle_mod.enginit_mesh(S.hist_struct(dict(ecdmin=ecdmin)), 1)
    assert len(uvcrd) == ermax and uvmax[0] == ermax and len(escrd) == esmax and uvsoft[0] == esmax
    assert np.all(np.diff(uvcrd) > 0)
    assert uvcrd[0] == pytest.approx(ecdmin - 10 * 2e-3)
    assert uvcrd[-1] == pytest.approx(1.0e11)


def test_binsearch_semantics(oracle_mod):
    c = [0.0, 1.0, 2.0]
    # returns the number of edges strictly below v (engproc.F90:1078-1108)
    assert oracle_mod.binsearch(c, -1.0) == 0
    assert oracle_mod.binsearch(c, 0.0) == 0      # equal to the first edge -> eng_min in getiduv
    assert oracle_mod.binsearch(c, 0.5) == 1
    assert oracle_mod.binsearch(c, 1.0) == 1
    assert oracle_mod.binsearch(c, 1.5) == 2
    assert oracle_mod.binsearch(c, 2.0) == 2
    assert oracle_mod.binsearch(c, 3.0) == 3
    rng = np.random.default_rng(0)
    e = np.sort(rng.normal(size=50))
    for v in rng.normal(size=200):
        assert oracle_mod.binsearch(e, v) == np.searchsorted(e, v, side="left")


@pytest.mark.parametrize("K,order", [(32, 6), (32, 4)])
def test_madelung_known_answer(oracle_mod, K, order):
    prm, topo, hist, pos, cell, ins, L = nacl_system(K=K, order=order)
    orc = oracle_mod.Oracle(prm, topo, hist)
    assert orc.engconst(1, pos, cell, ins_conf=ins) == 0
    u, u0 = orc.uvengy()
    d = 2.8
    e_int = COULOMB * (-MADELUNG_NACL / d - WIGNER_SC / L)
    e_self = 0.5 * COULOMB * WIGNER_SC / L
    assert u.sum() == pytest.approx(e_int, rel=2e-7)
    assert u0[0] == pytest.approx(e_self, rel=2e-7)


def test_lj_pair_analytic(oracle_mod):
    # two LJ sites at r < lwljcut: 4 eps ((s/r)^12 - (s/r)^6), no charges
    sg, ep, r = 3.4, 0.2, 3.9
    a = S.Species("a", np.zeros(1), np.array([sg]), np.array([ep]), np.array([12.0]), np.zeros((3, 1)))
    b = S.Species("b", np.zeros(1), np.array([sg]), np.array([ep]), np.array([12.0]), np.zeros((3, 1)))
    topo = S.Topology([a, b], [1, 1], [A.PT_SOLUTE, A.PT_SOLVENT])
    prm = S.default_params(slttype=A.SLT_SOLN, maxins=1, corrcal=0, wgtslf=0, ms1max=32)
    orc = oracle_mod.Oracle(prm, topo, dict(ecdmin=-20.0))
    pos = np.array([5.0, 5.0, 5.0, 5.0 + r, 5.0, 5.0], dtype=np.float32)
    cell = np.diag([30.0] * 3).astype(np.float32).ravel(order="F")
    assert orc.engconst(1, pos, cell) == 0
    u, _ = orc.uvengy()
    # the analytic value on the float32 inputs the reference's tables hold
    f = np.float32
    sg2 = float(f(((f(sg) + f(sg)) / f(2.0)) ** 2))
    e = float(np.sqrt(f(ep) * f(ep)))
    rr = float(f(5.0 + r) - f(5.0))
    x = (sg2 / rr ** 2) ** 3
    assert u[0, 1] == pytest.approx(4 * e * x * (x - 1), rel=1e-12)
    assert u[0, 0] == 0.0


def test_pme_self_energy_against_numpy(oracle_mod):
    """Recip self energy of a rigid ring = 1/2 sum engfac |rfftn(Q)|^2 with numpy's FFT."""
    w = S.make_workload(2, small=True, maxins=1)
    prm = dict(w.params, insposition=A.INSPOS_NOCHANGE, insorient=A.INSROT_NOCHANGE, slttype=A.SLT_REFS_FLEX,
               wgtslf=0)
    orc = oracle_mod.Oracle(prm, w.topo, w.hist)
    pos, cell = w.frame(0)
    conf = (w.topo.bfcoord.reshape(-1, 3) + 7.3).astype(np.float32)
    assert orc.engconst(1, pos, cell, ins_conf=conf.ravel()) == 0
    ef = orc.engfac()
    K = prm["ms1max"]
    L = float(np.float32(w.box))  # the cell arrives as float32
    # spread with the reference's spline rule (recpcal.F90:504-538, 453-473)
    n = prm["splodr"]
    Q = np.zeros((K, K, K))
    q = w.topo.charge[-w.topo.numsite[-1]:].astype(np.float64)
    for s, x in enumerate(conf.astype(np.float64)):
        u = (x / L) % 1.0 * K
        gi = np.floor(u).astype(int)
        wts = [[oracle_mod.spline_value(n, u[m] - (gi[m] - k)) for k in range(n)] for m in range(3)]
        for c3 in range(n):
            for c2 in range(n):
                for c1 in range(n):
                    Q[(gi[2] - c3) % K, (gi[1] - c2) % K, (gi[0] - c1) % K] += q[s] * wts[0][c1] * wts[1][c2] * wts[2][c3]
    F = np.fft.rfftn(Q)          # axes (z, y, x) with x halved: matches [K3][K2][K1/2+1]
    wgt = np.ones(K // 2 + 1)
    wgt[0] = wgt[-1] = 0.5
    self_np = float((ef * np.abs(F) ** 2 * wgt).sum())
    # uvengy0 = recip self + real self + residual; recover recip self by subtracting the analytic rest
    _, u0 = orc.uvengy()
    from math import erf, pi, sqrt
    al = float(np.float32(prm["screen"]))  # the C-ABI carries screen as float
    real = -np.sum(q ** 2) * al / sqrt(pi)
    for i in range(len(q)):
        for j in range(i + 1, len(q)):
            r = np.linalg.norm(conf[i].astype(np.float64) - conf[j])
            real -= q[i] * q[j] * erf(al * r) / r
    assert u0[0] - real == pytest.approx(self_np, rel=1e-9, abs=1e-9)


def test_engfac_symmetry(oracle_mod):
    w = S.make_workload(2, small=True, maxins=1)
    orc = oracle_mod.Oracle(w.params, w.topo, w.hist)
    pos, cell = w.frame(0)
    orc.engconst(1, pos, cell)
    ef = orc.engfac()
    K = w.params["ms1max"]
    assert ef[0, 0, 0] == 0.0
    # cubic box: invariant under k2 -> -k2, k3 -> -k3 and under exchange of axes 2 and 3
    assert np.allclose(ef, ef[::-1][np.r_[K - 1, 0:K - 1]][:, ::-1][:, np.r_[K - 1, 0:K - 1]], rtol=1e-12)
    assert np.allclose(ef, ef.transpose(1, 0, 2), rtol=1e-12)


def test_fp32_vs_fp64_oracle(oracle_mod):
    """The single-precision restatement stays within the stated energy tolerance of the FP64 one."""
    w = S.make_workload(2, small=True, maxins=8)
    o8 = oracle_mod.Oracle(w.params, w.topo, w.hist, precision=8)
    o4 = oracle_mod.Oracle(w.params, w.topo, w.hist, precision=4)
    pos, cell = w.frame(0)
    assert o8.engconst(1, pos, cell) >= 0 and o4.engconst(1, pos, cell) >= 0
    u8, _ = o8.uvengy()
    u4, _ = o4.uvengy()
    # soft region only: in the core region (E > 1e3 kcal/mol, overlapping atoms) E ~ r^-12
    # turns the FP32 placement rounding of the insertion into 1e-4-level relative differences
    soft = np.abs(u8) < 1.0e3
    assert soft.mean() > 0.9
    assert np.all(np.abs(u4 - u8)[soft] <= 1e-4 * np.abs(u8[soft]) + 1e-4)


def test_no_insertions_is_refused(oracle_mod):
    """maxins < 1 in refs mode halts with set_ins (setconf.F90:346-353)."""
    w = S.make_workload(2, small=True, maxins=8)
    with pytest.raises(RuntimeError, match="set_ins"):
        oracle_mod.Oracle(dict(w.params, maxins=0), w.topo, w.hist)
