"""PPPM (cltype 3): Hockney and Eastwood's optimal influence function in the oracle (CPU only).

The reference's PPPM shares spreading, FFT, gather and self terms with smooth PME
(engproc.F90:420-433) and differs only in the influence function
(recpcal_pppm_greenfunc, recpcal.F90:217-337).  Pins:
  * the alias-sum polynomial (calc_gfb_pppm, recpcal.F90:179-198) against the
    closed forms of Hockney and Eastwood and a direct sum over aliases,
  * the oracle's influence function against an independent numpy evaluation
    whose denominator is a direct alias sum rather than the polynomial,
  * the NaCl Madelung constant through the full realcal + PPPM chain,
  * agreement with smooth PME on a solvated system.
"""
import numpy as np
import pytest

from ermod_openacc_b200 import _capi as A
from ermod_openacc_b200 import systems as S
from _helpers import COULOMB, MADELUNG_NACL, WIGNER_SC, nacl_system

# sum_n (sin(pi t) / (pi (t + n)))^(2P) as polynomials in z = sin^2(pi t)
CLOSED_FORMS = {
    2: [1.0, -2.0 / 3.0],
    4: [1.0, -4.0 / 3.0, 2.0 / 5.0, -4.0 / 315.0],
}


@pytest.mark.parametrize("order", [2, 4])
def test_alias_polynomial_closed_forms(oracle_mod, order):
    assert np.allclose(oracle_mod.pppm_gfb(order), CLOSED_FORMS[order], rtol=1e-14, atol=1e-15)


@pytest.mark.parametrize("order", [2, 4, 6, 8])
def test_alias_polynomial_direct_sum(oracle_mod, order):
    b = oracle_mod.pppm_gfb(order)
    n = np.arange(-4000, 4001)
    for t in (0.05, 0.21, 0.37, 0.5):
        direct = np.sum((np.sin(np.pi * t) / (np.pi * (t + n))) ** (2 * order))
        z = np.sin(np.pi * t) ** 2
        assert np.polyval(b[::-1], z) == pytest.approx(direct, rel=1e-10)


def _mrange(cell_f, screen, K):
    """Alias range: float32 arithmetic and truncation as recpcal.F90:230-233."""
    f = np.float32
    acc = f(-np.log(f(1e-7))) ** f(0.25)
    mm = [f(screen) / (f(np.pi) * f(k)) * acc for k in K]
    return [int(f(cell_f[0, j] * mm[0] + cell_f[1, j] * mm[1] + cell_f[2, j] * mm[2])) for j in range(3)]


def _influence_numpy(cell, screen, K, order, mr):
    """G_opt on the [K3][K2][K1/2+1] half spectrum with the denominator as a direct alias sum."""
    inv = np.linalg.inv(cell.astype(np.float64))   # rows: reciprocal vectors (no 2 pi)
    vol = abs(np.linalg.det(cell.astype(np.float64)))
    K1, K2, K3 = K
    fold = lambda r, k: np.where(r <= k // 2, r, r - k).astype(np.float64)
    m1 = fold(np.arange(K1 // 2 + 1), K1)
    m2 = fold(np.arange(K2), K2)
    m3 = fold(np.arange(K3), K3)
    M3, M2, M1 = np.meshgrid(m3, m2, m1, indexing="ij")
    tp = 2.0 * np.pi

    def kvec(a, b, c):
        return [tp * (inv[i, 0] * a + inv[i, 1] * b + inv[i, 2] * c) for i in range(3)]

    def usq(m, k, n):
        t = np.pi * (m / k + n)
        with np.errstate(invalid="ignore", divide="ignore"):
            x = np.where(t == 0.0, 1.0, np.sin(t) / np.where(t == 0.0, 1.0, t))
        return x ** (2 * order)

    k = kvec(M1, M2, M3)
    k2 = k[0] ** 2 + k[1] ** 2 + k[2] ** 2
    num = np.zeros_like(k2)
    for nx in range(-mr[0], mr[0] + 1):
        for ny in range(-mr[1], mr[1] + 1):
            for nz in range(-mr[2], mr[2] + 1):
                km = kvec(M1 + nx * K1, M2 + ny * K2, M3 + nz * K3)
                kk = km[0] ** 2 + km[1] ** 2 + km[2] ** 2
                with np.errstate(invalid="ignore", divide="ignore"):
                    term = (k[0] * km[0] + k[1] * km[1] + k[2] * km[2]) * np.exp(-kk / (4 * screen ** 2)) \
                        * usq(M1, K1, nx) * usq(M2, K2, ny) * usq(M3, K3, nz) / kk
                num += np.nan_to_num(term)
    nn = np.arange(-3000, 3001)
    den = np.ones_like(k2)
    for m, kk in ((M1, K1), (M2, K2), (M3, K3)):
        t = m / kk
        s = np.zeros_like(t)
        for n in nn:
            tt = np.pi * (t + n)
            with np.errstate(invalid="ignore", divide="ignore"):
                s += np.where(tt == 0.0, 1.0, (np.sin(np.pi * t) / np.where(tt == 0.0, 1.0, tt)) ** (2 * order))
        den *= s
    with np.errstate(invalid="ignore", divide="ignore"):
        g = num * 4.0 * np.pi / (k2 * den ** 2) / vol
    g[0, 0, 0] = 0.0
    return g


def _pppm_workload(ms, order, box_scale=1.0):
    w = S.make_workload(2, small=True, maxins=4)
    prm = dict(w.params, cltype=A.EL_PPPM, splodr=order, ms1max=ms[0], ms2max=ms[1], ms3max=ms[2])
    pos, cell = w.frame(0)
    return w, prm, pos, cell


@pytest.mark.parametrize("ms,order,screen", [((32, 32, 32), 4, None), ((12, 16, 10), 6, 0.9), ((8, 8, 12), 4, 1.2)])
def test_influence_function_against_numpy(oracle_mod, ms, order, screen):
    w, prm, pos, cell = _pppm_workload(ms, order)
    if screen is not None:
        prm["screen"] = screen
    orc = oracle_mod.Oracle(prm, w.topo, w.hist)
    assert orc.engconst(1, pos, cell) == 0, orc.last_error()
    ef = orc.engfac()
    c = np.asarray(cell, dtype=np.float32).reshape(3, 3, order="F")
    scr = float(np.float32(prm["screen"]))
    mr = _mrange(c, scr, ms)
    if screen is not None and screen >= 0.9:
        assert max(mr) >= 1          # the coarse meshes exercise the alias sums
    g = _influence_numpy(c, scr, ms, order, mr)
    assert ef.shape == g.shape
    assert np.allclose(ef, g, rtol=1e-9, atol=1e-14 * np.abs(g).max())


def _madelung_errors(oracle_mod, K, order):
    prm, topo, hist, pos, cell, ins, L = nacl_system(K=K, order=order)
    prm = dict(prm, cltype=A.EL_PPPM)
    orc = oracle_mod.Oracle(prm, topo, hist)
    assert orc.engconst(1, pos, cell, ins_conf=ins) == 0
    u, u0 = orc.uvengy()
    d = 2.8
    e_int = COULOMB * (-MADELUNG_NACL / d - WIGNER_SC / L)
    e_self = 0.5 * COULOMB * WIGNER_SC / L
    return abs(u.sum() / e_int - 1.0), abs(u0[0] / e_self - 1.0)


@pytest.mark.parametrize("K,order,tol", [(32, 6, 5e-6), (32, 8, 5e-7), (64, 6, 5e-7)])
def test_madelung_known_answer_pppm(oracle_mod, K, order, tol):
    """The force-optimised influence function carries an energy bias that falls fast with order."""
    e_int, e_self = _madelung_errors(oracle_mod, K, order)
    assert e_int < tol and e_self < tol


def test_madelung_pppm_converges(oracle_mod):
    """Order 4: the lattice-energy error falls with the mesh spacing (32 -> 64 points)."""
    coarse = _madelung_errors(oracle_mod, 32, 4)
    fine = _madelung_errors(oracle_mod, 64, 4)
    assert coarse[0] < 1e-4 and coarse[1] < 5e-4
    assert fine[0] < coarse[0] / 8 and fine[1] < coarse[1] / 8


def test_pppm_close_to_pme(oracle_mod):
    """On a fine mesh both mesh methods approach Ewald: per-molecule energies agree closely."""
    w = S.make_workload(2, small=True, maxins=8)
    pos, cell = w.frame(0)
    out = {}
    for cl in (A.EL_PME, A.EL_PPPM):
        prm = dict(w.params, cltype=cl, splodr=6)
        orc = oracle_mod.Oracle(prm, w.topo, w.hist)
        assert orc.engconst(1, pos, cell) == 0
        out[cl] = orc.uvengy()
    u_pme, u0_pme = out[A.EL_PME]
    u_pppm, u0_pppm = out[A.EL_PPPM]
    assert np.abs(u_pppm - u_pme).max() < 2e-4
    assert np.allclose(u0_pppm, u0_pme, atol=2e-4)


def test_pppm_odd_order_rejected(oracle_mod):
    w = S.make_workload(2, small=True, maxins=4)
    prm = dict(w.params, cltype=A.EL_PPPM, splodr=5)
    with pytest.raises(Exception):
        oracle_mod.Oracle(prm, w.topo, w.hist)
