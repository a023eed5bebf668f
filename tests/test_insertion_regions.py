"""Insertion regions (insposition 2..4, insertion.F90:164-200) on the CPU oracle.

The solute's centre of mass goes first to the mass-weighted centre of the host
aggregate (insorigin 2, com_aggregate insertion.F90:587-614), then:
  sphere (2):          + a point of the shell lwreg <= r <= upreg, uniform in volume
  slab generic (3):    + cell . (u1, u2, dz / |c3|), lwreg <= dz <= upreg
  slab symmetric (4):  the same with dz of either sign, each with probability 1/2
These tests check those geometries and distributions on the oracle's own
placements; tests/test_parity_gpu.py checks the GPU's placements against it.
"""
import numpy as np
import pytest

from ermod_openacc_b200 import _capi as A
from ermod_openacc_b200 import systems as S

NINS = 2000


def aggregate_center(topo, pos, hostspec):
    xyz = np.asarray(pos, dtype=np.float64).reshape(-1, 3)
    mb = np.concatenate([[0], np.cumsum(topo.numsite)])
    num, den = np.zeros(3), 0.0
    for i in range(len(topo.numsite)):
        sp = int(topo.uvspec[i])
        if topo.sluvid[i] != A.PT_SOLVENT or sp < 1 or not (hostspec >> (sp - 1)) & 1:
            continue
        m = topo.sitemass[mb[i]:mb[i + 1]].astype(np.float64)
        num += (m[:, None] * xyz[mb[i]:mb[i + 1]]).sum(axis=0)
        den += m.sum()
    return num / den


def placements(oracle_mod, insposition, lwreg, upreg, insorient=A.INSROT_RANDOM, maxins=NINS, periodic=True):
    w = S.make_workload(2, small=True, maxins=maxins)
    prm = dict(w.params, insposition=insposition, insorient=insorient, lwreg=lwreg, upreg=upreg, hostspec=1,
               corrcal=0)
    orc = oracle_mod.Oracle(prm, w.topo, w.hist)
    pos, cell = w.frame(0)
    assert orc.engconst(1, pos, cell) >= 0
    s = int(w.topo.numsite[-1])
    ins = np.asarray(orc.insertions(), dtype=np.float64).reshape(maxins, s, 3)
    m = w.topo.sitemass[-s:].astype(np.float64)
    com = (ins * m[None, :, None]).sum(axis=1) / m.sum()
    return com, aggregate_center(w.topo, pos, 1), np.asarray(cell, dtype=np.float64).reshape(3, 3)


def test_sphere_shell_uniform_in_volume(oracle_mod):
    lw, up = 3.0, 8.0
    com, ag, _ = placements(oracle_mod, A.INSPOS_SPHERE, lw, up)
    r = np.linalg.norm(com - ag, axis=1)
    assert r.min() >= lw - 1e-3 and r.max() <= up + 1e-3
    # uniform in volume: F(r) = (r^3 - lw^3) / (up^3 - lw^3); Kolmogorov-Smirnov distance
    rs = np.sort(r)
    F = (rs ** 3 - lw ** 3) / (up ** 3 - lw ** 3)
    ecdf = np.arange(1, len(rs) + 1) / len(rs)
    assert np.max(np.abs(ecdf - F)) < 1.63 / np.sqrt(len(rs))   # 1% level
    # isotropic directions: the mean unit vector is near zero
    u = (com - ag) / r[:, None]
    assert np.linalg.norm(u.mean(axis=0)) < 4.0 / np.sqrt(len(rs))


@pytest.mark.parametrize("insposition", [A.INSPOS_SLAB_GENERIC, A.INSPOS_SLAB_SYMMETRIC])
def test_slab_offsets(oracle_mod, insposition):
    lw, up = 2.0, 6.0
    com, ag, cell = placements(oracle_mod, insposition, lw, up)
    dz = com[:, 2] - ag[2]                     # cuboid cell: the third cell vector is along z
    a = np.abs(dz)
    assert a.min() >= lw - 1e-3 and a.max() <= up + 1e-3
    if insposition == A.INSPOS_SLAB_GENERIC:
        assert np.all(dz > 0)
    else:
        frac_neg = (dz < 0).mean()
        assert abs(frac_neg - 0.5) < 4 * 0.5 / np.sqrt(len(dz))
    # x and y cover the cell uniformly from the aggregate centre
    for k in (0, 1):
        f = (com[:, k] - ag[k]) / cell[k, k]
        assert f.min() >= -1e-6 and f.max() <= 1 + 1e-6
        assert abs(f.mean() - 0.5) < 4 * np.sqrt(1 / 12) / np.sqrt(len(f))


def test_region_without_rotation_keeps_the_body_frame(oracle_mod):
    """insorient 1: only the COM moves; the solute keeps its body-fixed orientation."""
    w = S.make_workload(2, small=True, maxins=16)
    prm = dict(w.params, insposition=A.INSPOS_SPHERE, insorient=A.INSROT_NOCHANGE, lwreg=0.0, upreg=5.0,
               hostspec=1, corrcal=0)
    orc = oracle_mod.Oracle(prm, w.topo, w.hist)
    pos, cell = w.frame(0)
    assert orc.engconst(1, pos, cell) >= 0
    s = int(w.topo.numsite[-1])
    ins = np.asarray(orc.insertions(), dtype=np.float64).reshape(16, s, 3)
    bf = np.asarray(w.topo.bfcoord, dtype=np.float64).reshape(s, 3)
    m = w.topo.sitemass[-s:].astype(np.float64)
    bf_c = bf - (bf * m[:, None]).sum(axis=0) / m.sum()
    for c in range(16):
        rel = ins[c] - (ins[c] * m[:, None]).sum(axis=0) / m.sum()
        np.testing.assert_allclose(rel, bf_c, atol=1e-6)


def test_region_parameters_are_checked(oracle_mod):
    w = S.make_workload(2, small=True, maxins=8)
    for bad in (dict(hostspec=0, lwreg=1.0, upreg=2.0), dict(hostspec=1, lwreg=3.0, upreg=2.0),
                dict(hostspec=1, lwreg=0.0, upreg=0.0)):
        prm = dict(w.params, insposition=A.INSPOS_SPHERE, **bad)
        with pytest.raises(Exception):
            oracle_mod.Oracle(prm, w.topo, w.hist)


# ---- solutes in solution: check_mol_configuration (engproc.F90:1197-1324) ----
from _helpers import soln_multi_system  # noqa: E402


@pytest.mark.parametrize("insposition,lw,up,expect", [
    (A.INSPOS_SPHERE, 3.0, 8.0, [False, True, True, False]),          # |offset| 1.5, 5, 7, 10
    (A.INSPOS_SLAB_SYMMETRIC, 8.0, 11.0, [False, False, False, True]), # |dz| 0, 0, 0, 10
    (A.INSPOS_SLAB_GENERIC, 8.0, 11.0, [False, False, False, False]),  # dz = -10 is below the slab
    (A.INSPOS_RANDOM, 0.0, 0.0, [True, True, True, True]),
])
def test_soln_configuration_check(oracle_mod, insposition, lw, up, expect):
    """A solute whose centre of mass lies outside the region around the water aggregate's centre
    is skipped for the frame: no energies and no update_histogram (engproc.F90:447-450, 754-755)."""
    prm, topo, hist, pos, cell, _ = soln_multi_system()
    prm = dict(prm, insposition=insposition, lwreg=lw, upreg=up, keep_uvengy=1)
    orc = oracle_mod.Oracle(prm, topo, hist)
    assert orc.engconst(1, pos, cell) >= 0
    u, _ = orc.uvengy()
    kept = np.array(expect)
    assert np.all(np.any(u[kept] != 0.0, axis=1))
    assert np.all(u[~kept] == 0.0)
    a = orc.accum()
    assert a["engsmpl"] == kept.sum()
    # each kept solute bins every other molecule once, with the same weight (neutral solutes)
    assert a["edens"].sum() == pytest.approx(a["engnorm"] * (u.shape[1] - 1), rel=1e-9, abs=1e-12)


# ---- RMSD / Gaussian insertion against the RefInfo structure (insorigin 3) ----
def _rot(axis, ang):
    axis = np.asarray(axis, dtype=np.float64) / np.linalg.norm(axis)
    K = np.array([[0, -axis[2], axis[1]], [axis[2], 0, -axis[0]], [-axis[1], axis[0], 0]])
    return np.eye(3) + np.sin(ang) * K + (1 - np.cos(ang)) * K @ K


def refinfo_case(maxins=256):
    """The C2 small workload with a RefInfo whose host is this frame's water moved by a known rigid
    motion M, and whose solute is M applied to a known placement slt0 of the ring: reffit must
    carry the reference solute back onto slt0."""
    w = S.make_workload(2, small=True, maxins=maxins)
    pos, cell = w.frame(0)
    xyz = np.asarray(pos, dtype=np.float64).reshape(-1, 3)
    R, t = _rot([1.0, 2.0, -0.5], 0.7), np.array([3.0, -4.0, 1.5])
    host_ref = xyz @ R.T + t
    s = int(w.topo.numsite[-1])
    bf = np.asarray(w.topo.bfcoord, dtype=np.float64).reshape(s, 3)
    slt0 = bf - bf.mean(axis=0) + np.array([12.0, 13.0, 11.0])
    slt_ref = slt0 @ R.T + t
    ref = dict(refspec=1, host_crd=host_ref.ravel(), host_w=np.ones(len(xyz)), slt_crd=slt_ref.ravel(),
               slt_w=np.ones(s))
    return w, pos, cell, ref, slt0


def _rmsd(a, b):
    return np.sqrt(((a - b) ** 2).sum(axis=-1).mean(axis=-1))


@pytest.mark.parametrize("insorient", [A.INSROT_NOCHANGE, A.INSROT_RANDOM])
def test_rmsd_insertion_window(oracle_mod, insorient):
    w, pos, cell, ref, slt0 = refinfo_case()
    lw, up = 1.0, 4.0
    prm = dict(w.params, insposition=A.INSPOS_RMSD, insorient=insorient, lwreg=lw, upreg=up, corrcal=0)
    orc = oracle_mod.Oracle(prm, w.topo, w.hist)
    orc.set_refstructure(**ref)
    assert orc.engconst(1, pos, cell) >= 0
    s = slt0.shape[0]
    ins = np.asarray(orc.insertions(), dtype=np.float64).reshape(-1, s, 3)
    r = _rmsd(ins, slt0[None])
    assert r.min() >= lw - 1e-3 and r.max() <= up + 1e-3
    if insorient == A.INSROT_NOCHANGE:   # a pure translation of the fitted reference: rigid copies of slt0
        rel = ins - ins.mean(axis=1, keepdims=True)
        np.testing.assert_allclose(rel, np.broadcast_to(slt0 - slt0.mean(axis=0), rel.shape), atol=2e-4)
    assert np.all(orc.insertion_weights() == 1.0)


def test_gaussian_insertion_weights(oracle_mod):
    """Mixture of uniform and Gaussian displacements: each weight is 1/q of the mixture density, so
    with every first try accepted (a wide RMSD window) the weights average z0 = 8 l1 l2 l3."""
    w, pos, cell, ref, slt0 = refinfo_case(maxins=4000)
    up = 40.0
    prm = dict(w.params, insposition=A.INSPOS_GAUSS, lwreg=0.0, upreg=up, corrcal=0)
    orc = oracle_mod.Oracle(prm, w.topo, w.hist)
    orc.set_refstructure(**ref)
    assert orc.engconst(1, pos, cell) >= 0
    wt = orc.insertion_weights()
    L = np.linalg.norm(np.asarray(cell, dtype=np.float64).reshape(3, 3), axis=0)
    l = (L / 2) / up
    assert np.all(np.isfinite(wt)) and np.all(wt > 0)
    assert abs(wt.mean() / (8 * np.prod(l)) - 1.0) < 0.1


def test_soln_rmsd_check(oracle_mod):
    """Solutes in solution with insposition 5: kept when their RMSD to the best-fit reference
    solute lies in lwreg..upreg (engproc.F90:1249-1269)."""
    from _helpers import soln_multi_system
    prm, topo, hist, pos, cell, offs = soln_multi_system()
    xyz = np.asarray(pos, dtype=np.float64).reshape(-1, 3)
    nslt = len(offs)
    water = xyz[nslt:]
    R, t = _rot([0.3, -1.0, 0.2], 1.1), np.array([-2.0, 1.0, 5.0])
    ref = dict(refspec=2, host_crd=(water @ R.T + t).ravel(), host_w=np.ones(len(water)),
               slt_crd=(xyz[1:2] @ R.T + t).ravel(), slt_w=np.ones(1))
    prm = dict(prm, insposition=A.INSPOS_RMSD, lwreg=0.0, upreg=1.0, keep_uvengy=1)
    orc = oracle_mod.Oracle(prm, topo, hist)
    orc.set_refstructure(**ref)
    assert orc.engconst(1, pos, cell) >= 0
    u, _ = orc.uvengy()
    np.testing.assert_array_equal(np.any(u != 0.0, axis=1), [False, True, False, False])
    assert orc.accum()["engsmpl"] == 1


def _structure_case(lw, up, **extra):
    from _helpers import soln_struct_system
    prm, topo, hist, pos, cell, ideal, wts = soln_struct_system()
    xyz = np.asarray(pos, dtype=np.float64).reshape(-1, 3)
    water = xyz[12:]
    prm = dict(prm, insstructure=A.INSSTR_RMSD, lwstr=lw, upstr=up, keep_uvengy=1, **extra)
    ref = dict(refspec=2, host_crd=water.ravel(), host_w=np.ones(len(water)), slt_crd=ideal.ravel(), slt_w=wts)
    return prm, topo, hist, pos, cell, ref, xyz[:12].reshape(4, 3, 3), ideal, wts


def _kabsch(ref, x, w):
    cr = (w[:, None] * ref).sum(0) / w.sum()
    cx = (w[:, None] * x).sum(0) / w.sum()
    U, _, Vt = np.linalg.svd(((x - cx) * w[:, None]).T @ (ref - cr))
    R = Vt.T @ np.diag([1.0, 1.0, np.sign(np.linalg.det(Vt.T @ U.T))]) @ U.T
    return float(np.sqrt((w * (((x - cx) @ R.T + cr - ref) ** 2).sum(1)).sum() / w.sum()))


def test_soln_structure_check(oracle_mod):
    """insstructure 1 in solution: a solute whose best-fit RMSD from RefInfo's solute lies
    outside lwstr..upstr is skipped for the frame (engproc.F90:1277-1295)."""
    prm, topo, hist, pos, cell, ref, slts, ideal, wts = _structure_case(0.0, 0.05)
    rms = np.array([_kabsch(ideal, g, wts) for g in slts])     # mass weights: 0, 0.016, 0.094, 0.188
    keep = (rms >= 0.0) & (rms <= 0.05)
    assert keep.tolist() == [True, True, False, False]
    assert np.all(np.abs(rms - 0.05) > 0.03)
    orc = oracle_mod.Oracle(prm, topo, hist)
    assert orc.engconst(1, pos, cell) < 0                       # RefInfo is required
    assert orc.last_error() == "ins_ref"
    orc = oracle_mod.Oracle(prm, topo, hist)
    orc.set_refstructure(**ref)
    assert orc.engconst(1, pos, cell) >= 0
    u, _ = orc.uvengy()
    np.testing.assert_array_equal(np.any(u != 0.0, axis=1), keep)
    assert orc.accum()["engsmpl"] == keep.sum()
    # lower bound only: the two distorted solutes
    prm2, *_ = _structure_case(0.05, 10.0)
    orc = oracle_mod.Oracle(prm2, topo, hist)
    orc.set_refstructure(**ref)
    assert orc.engconst(1, pos, cell) >= 0
    np.testing.assert_array_equal(np.any(orc.uvengy()[0] != 0.0, axis=1), ~keep)
    # with the sphere window as well: both checks apply (the region first)
    prm3, *_ = _structure_case(0.0, 0.05, insposition=A.INSPOS_SPHERE, lwreg=0.0, upreg=3.0)
    orc = oracle_mod.Oracle(prm3, topo, hist)
    orc.set_refstructure(**ref)
    assert orc.engconst(1, pos, cell) >= 0
    near = np.linalg.norm(slts.mean(axis=1) - 24.9 / 2, axis=1) < 3.0
    np.testing.assert_array_equal(np.any(orc.uvengy()[0] != 0.0, axis=1), keep & near)


def test_unknown_insstructure_is_refused(oracle_mod):
    prm, topo, hist, *_ = _structure_case(0.0, 0.1)
    with pytest.raises(RuntimeError, match="ins_str"):
        oracle_mod.Oracle(dict(prm, insstructure=2), topo, hist)


def test_refstructure_is_required(oracle_mod):
    w = S.make_workload(2, small=True, maxins=8)
    prm = dict(w.params, insposition=A.INSPOS_RMSD, lwreg=0.0, upreg=4.0)
    orc = oracle_mod.Oracle(prm, w.topo, w.hist)
    pos, cell = w.frame(0)
    assert orc.engconst(1, pos, cell) < 0
