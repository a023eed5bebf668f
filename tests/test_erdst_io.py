"""erdst's on-disk formats through the library (CPU only): DCD reading, engstore's files,
the Fortran edit descriptors they use, rmsd_bestfit, and the file round trip into slvfe."""
import os

import numpy as np
import pytest

from ermod_openacc_b200 import _capi as A
from ermod_openacc_b200 import erdst_io as IO
from ermod_openacc_b200 import slvfe as SF
from ermod_openacc_b200 import systems as S
from _dcd import cell_record, vmd_cell, write_dcd

# ---------------------------------------------------------------------------
# Fortran edit descriptors (F2008 10.7.2.3, 10.7.5.2.2), fields worked out by hand:
# G: F(w-4).(d-k) + 4 blanks when 0.1 <= |x| < 10^d after rounding to d digits, k the
# decimal exponent; zero as F(w-4).(d-1); E editing otherwise, with a three-digit
# exponent written without the letter.
# ---------------------------------------------------------------------------
FORMAT_CASES = [
    ("G", 1.5, 15, 7, "   1.500000    "),
    ("G", 0.0, 15, 7, "   0.000000    "),
    ("G", 123.456, 15, 7, "   123.4560    "),
    ("G", 0.5, 15, 7, "  0.5000000    "),
    ("G", -0.05, 15, 7, " -0.5000000E-01"),
    ("G", 12345678.0, 15, 7, "  0.1234568E+08"),
    ("G", 9999999.6, 15, 7, "  0.1000000E+08"),     # rounds up to 10^7: E editing
    ("G", 0.09999999996, 15, 7, "  0.1000000    "),  # rounds up to 0.1: F editing
    ("G", 1e-120, 15, 7, "  0.1000000-119"),
    ("G", -20.0, 15, 7, "  -20.00000    "),
    ("G", 1.0 / 3.0, 25, 15, "    0.333333333333333    "),
    ("G", 2.5e-7, 25, 15, "    0.250000000000000E-06"),
    ("G", 1.5e5, 18, 5, "       0.15000E+06"),
    ("G", 99999.0, 18, 5, "        99999.    "),
    ("E", 1.0, 20, 8, "      0.10000000E+01"),
    ("E", -123.456, 20, 7, "      -0.1234560E+03"),
    ("E", 0.0, 20, 8, "      0.00000000E+00"),
    ("F", -3.14159265, 15, 5, "       -3.14159"),
    ("F", 0.25, 15, 5, "        0.25000"),
    ("F", 1e12, 15, 5, "***************"),
    ("I", 12, 5, 0, "   12"),
    ("I", 123456, 5, 0, "*****"),
]


@pytest.mark.parametrize("kind,x,w,d,want", FORMAT_CASES)
def test_fortran_edit_descriptors(engine_lib, kind, x, w, d, want):
    assert IO.fortran_format(kind, x, w, d) == want


def test_leading_zero_dropped_only_when_one_short(engine_lib):
    # -0.1234567E+01 is 14 characters: it fits E14.7 as is, E13.7 drops the zero, E12.7 overflows
    assert IO.fortran_format("E", -1.234567, 14, 7) == "-0.1234567E+01"
    assert IO.fortran_format("E", -1.234567, 13, 7) == "-.1234567E+01"
    assert IO.fortran_format("E", -1.234567, 12, 7) == "*" * 12


# ---------------------------------------------------------------------------
# DCD reading
# ---------------------------------------------------------------------------
def _frames(n=5, natoms=7, seed=3):
    rng = np.random.default_rng(seed)
    return [rng.uniform(-5, 30, size=(natoms, 3)).astype(np.float32) for _ in range(n)]


@pytest.mark.parametrize("end,marker", [("<", 4), (">", 4), ("<", 8), (">", 8)])
def test_dcd_byte_orders_and_markers(engine_lib, tmp_path, end, marker):
    fr = _frames()
    cells = [cell_record(30.0 + k, 31.0, 32.0, 90.0, 90.0, 90.0) for k in range(len(fr))]
    p = tmp_path / "h.dcd"
    write_dcd(p, fr, cells, end=end, marker=marker)
    with IO.Trajectory(p) as t:
        assert (t.natoms, t.nframes, t.has_cell) == (7, 5, True)
        for k in range(5):
            crd, cell = t.read()
            np.testing.assert_array_equal(crd.reshape(-1, 3), fr[k])
            np.testing.assert_allclose(cell, vmd_cell(30.0 + k, 31.0, 32.0, 90.0, 90.0, 90.0), atol=1e-5)
            assert cell[1] == cell[2] == cell[5] == 0.0
        assert t.read() is None


@pytest.mark.parametrize("cosines", [True, False])
def test_dcd_triclinic_cell(engine_lib, tmp_path, cosines):
    """Angle cosines (CHARMM, NAMD >= 2.5) and degrees (NAMD 2.5) give the same cell."""
    fr = _frames(2)
    par = (40.0, 42.0, 45.0, 70.0, 80.0, 100.0)
    p = tmp_path / "t.dcd"
    write_dcd(p, fr, [cell_record(*par, cosines=cosines)] * 2)
    with IO.Trajectory(p) as t:
        _, cell = t.read()
    want = vmd_cell(*par)
    np.testing.assert_allclose(cell, want, rtol=2e-6, atol=2e-5)
    # the three vectors keep their lengths and angles
    a, b, c = cell[0:3].astype(float), cell[3:6].astype(float), cell[6:9].astype(float)
    assert np.linalg.norm(b) == pytest.approx(42.0, rel=1e-6)
    ang = lambda u, v: np.degrees(np.arccos(np.dot(u, v) / np.linalg.norm(u) / np.linalg.norm(v)))
    assert ang(b, c) == pytest.approx(70.0, abs=1e-4)
    assert ang(a, c) == pytest.approx(80.0, abs=1e-4)
    assert ang(a, b) == pytest.approx(100.0, abs=1e-4)


def test_dcd_xplor_and_4d(engine_lib, tmp_path):
    fr = _frames(3)
    p = tmp_path / "x.dcd"
    write_dcd(p, fr, None, charmm=False)
    with IO.Trajectory(p) as t:
        assert not t.has_cell
        crd, cell = t.read()
        np.testing.assert_array_equal(crd.reshape(-1, 3), fr[0])
        assert not cell.any()
    q = tmp_path / "d4.dcd"
    write_dcd(q, fr, [cell_record(20, 20, 20, 90, 90, 90)] * 3, dim4=True)
    with IO.Trajectory(q) as t:
        got = [t.read() for _ in range(4)]
    assert got[3] is None
    np.testing.assert_array_equal(got[2][0].reshape(-1, 3), fr[2])


def test_dcd_rewind_and_header_count(engine_lib, tmp_path):
    fr = _frames(3)
    p = tmp_path / "r.dcd"
    write_dcd(p, fr, None, nframes=0)        # a writer that never filled in NSET
    with IO.Trajectory(p) as t:
        assert t.nframes == 0
        for _ in range(3):
            assert t.read() is not None
        assert t.read() is None
        t.rewind()
        np.testing.assert_array_equal(t.read()[0].reshape(-1, 3), fr[0])


def test_dcd_errors(engine_lib, tmp_path):
    fr = _frames(2)
    with pytest.raises(IO.IOError_, match="trj_opn"):
        IO.Trajectory(tmp_path / "missing.dcd")
    bad = tmp_path / "bad.dcd"
    bad.write_bytes(b"not a trajectory file at all" * 4)
    with pytest.raises(IO.IOError_, match="trj_hdr"):
        IO.Trajectory(bad)
    fx = tmp_path / "fixed.dcd"
    write_dcd(fx, fr, None, fixed=2)
    with pytest.raises(IO.IOError_, match="trj_fix"):
        IO.Trajectory(fx)
    tr = tmp_path / "trunc.dcd"
    write_dcd(tr, fr, [cell_record(20, 20, 20, 90, 90, 90)] * 2, truncate=10)
    with IO.Trajectory(tr) as t:
        assert t.read() is not None
        with pytest.raises(IO.IOError_, match="trj_rec"):
            t.read()
    ok = tmp_path / "ok.dcd"
    write_dcd(ok, fr, None)
    with IO.Trajectory(ok) as t:
        with pytest.raises(IO.IOError_, match="trj_nat"):
            t.read(natoms=6)


# ---------------------------------------------------------------------------
# rmsd_bestfit
# ---------------------------------------------------------------------------
def _kabsch_rmsd(ref, x, w):
    w = np.asarray(w, dtype=np.float64)
    cr = (w[:, None] * ref).sum(0) / w.sum()
    cx = (w[:, None] * x).sum(0) / w.sum()
    H = ((x - cx) * w[:, None]).T @ (ref - cr)
    U, _, Vt = np.linalg.svd(H)
    dd = np.sign(np.linalg.det(Vt.T @ U.T))
    R = Vt.T @ np.diag([1.0, 1.0, dd]) @ U.T
    y = (x - cx) @ R.T + cr
    return float(np.sqrt((w * ((y - ref) ** 2).sum(1)).sum() / w.sum()))


def test_rmsd_bestfit(engine_lib):
    rng = np.random.default_rng(5)
    ref = rng.normal(scale=3.0, size=(12, 3))
    w = rng.uniform(1.0, 16.0, size=12)
    q = rng.normal(size=4)
    q /= np.linalg.norm(q)
    a, b, c, d = q
    R = np.array([[a * a + b * b - c * c - d * d, 2 * (b * c - a * d), 2 * (b * d + a * c)],
                  [2 * (b * c + a * d), a * a - b * b + c * c - d * d, 2 * (c * d - a * b)],
                  [2 * (b * d - a * c), 2 * (c * d + a * b), a * a - b * b - c * c + d * d]])
    moved = ref @ R.T + np.array([4.0, -2.0, 7.5])
    assert IO.rmsd_bestfit(ref, moved, w) < 1e-5
    noisy = moved + rng.normal(scale=0.3, size=moved.shape)
    assert IO.rmsd_bestfit(ref, noisy, w) == pytest.approx(_kabsch_rmsd(ref, noisy, w), rel=1e-5)
    with pytest.raises(IO.IOError_, match="bst_zrw"):
        IO.rmsd_bestfit(ref, noisy, np.zeros(12))


# ---------------------------------------------------------------------------
# engstore's files and the round trip into slvfe
# ---------------------------------------------------------------------------
def _oracle_division(oracle_mod, w, prm, topo, frames, ins_seed=0):
    orc = oracle_mod.Oracle(prm, topo, w.hist, precision=8)
    for fr in range(frames):
        pos, cell = w.frame(fr)
        assert orc.engconst(fr + 1, pos, cell) >= 0
    raw = orc.accum()
    norm = orc.accum(normalise=True)
    kT = prm["temp"]
    sgn = -1.0 if prm["slttype"] == A.SLT_SOLN else 1.0
    avediv = np.array([[raw["engnorm"] / raw["engsmpl"], raw["voffset"] + sgn * kT * np.log(norm["avslf"])]])
    mesh = dict(uvcrd=orc.uvcrd, uvmax=orc.uvmax, uvsoft=orc.uvsoft, escrd=orc.escrd)
    return orc, norm, avediv, mesh


def _soln_and_refs(oracle_mod, tmp_path):
    w = S.make_workload(1, small=True)
    prm_s = dict(w.params, selfcal=0)
    orc_s, norm_s, av_s, mesh_s = _oracle_division(oracle_mod, w, prm_s, w.topo, 3)
    topo = S.Topology([S.water(), S.lj_site()], [w.nside ** 3, 1], [A.PT_SOLVENT, A.PT_TEST_RIGID])
    prm_r = S.default_params(ms1max=32, maxins=3000, selfcal=1)
    wr = S.Workload("refs-ljsite", prm_r, topo, w.hist, w.box, w.nside, 4, w.seed + 11)
    orc_r, norm_r, av_r, mesh_r = _oracle_division(oracle_mod, wr, prm_r, topo, 4)
    sd, rd = tmp_path / "soln", tmp_path / "refs"
    sd.mkdir()
    rd.mkdir()
    aveuv = norm_s["slnuv"].reshape(1, -1)
    IO.write_engstore(sd, prm_s, mesh_s, norm_s, 1, 1, av_s, aveuv)
    IO.write_engstore(rd, prm_r, mesh_r, norm_r, 1, 1, av_r)
    return (orc_s, norm_s, av_s, mesh_s, sd), (orc_r, norm_r, av_r, mesh_r, rd)


def test_engstore_files(engine_lib, oracle_mod, tmp_path):
    (orc_s, norm_s, av_s, mesh_s, sd), (orc_r, norm_r, av_r, mesh_r, rd) = _soln_and_refs(oracle_mod, tmp_path)
    want_s = ["aveuv.tt", "engsln.tt", "uvrange.tt", "weight_soln"] + (["corsln.tt"] if orc_s.params["corrcal"] else [])
    assert sorted(os.listdir(sd)) == sorted(want_s)
    assert sorted(os.listdir(rd)) == ["corref.tt", "engref.tt", "slfeng.tt", "uvrange.tt", "weight_refs"]
    lines = open(rd / "engref.tt").read().splitlines()
    assert lines[0] == "#      bin_left     bin_middle spec                    ratio                     dens"
    assert len(lines) == orc_r.ermax + 1 and all(len(l) == 85 for l in lines[1:])
    e = SF.read_engfile(rd / "engref.tt")
    left, middle, invwt, spec = SF.representative_bins(mesh_r["uvcrd"], mesh_r["uvmax"], mesh_r["uvsoft"])
    np.testing.assert_allclose(e["ratio"], norm_r["edens"], rtol=1e-14, atol=1e-300)
    np.testing.assert_allclose(e["dens"], norm_r["edens"] * invwt, rtol=1e-14, atol=1e-300)
    np.testing.assert_allclose(e["left"], left, rtol=5.01e-7)   # 7 significant digits
    np.testing.assert_allclose(e["middle"], middle, rtol=5.01e-7)
    np.testing.assert_array_equal(e["spec"], spec)
    chi = SF.read_corfile(rd / "corref.tt", orc_r.ermax)
    np.testing.assert_array_equal(chi, norm_r["ecorr"].T)
    assert os.path.getsize(rd / "corref.tt") == orc_r.ermax ** 2 * 8 + 8
    wr = open(rd / "weight_refs").read().splitlines()
    assert len(wr) == 1 and len(wr[0]) == 45 and wr[0].startswith("    1")
    t = SF.read_table(rd / "weight_refs")
    assert t[0, 1] == pytest.approx(av_r[0, 0], rel=5.01e-8)   # e20.8
    assert t[0, 2] == pytest.approx(av_r[0, 1], rel=5.01e-7)   # e20.7
    ws = open(sd / "weight_soln").read().splitlines()
    assert len(ws) == 1 and len(ws[0]) == 25 + 20 * orc_s.params["wgtslf"]   # (i5,e20.8[,e20.7])
    uv = open(rd / "uvrange.tt").read().splitlines()
    assert uv[0] == " species     minimum        maximum" and len(uv) == orc_r.numslv + 2
    u = SF.read_table(rd / "uvrange.tt")
    np.testing.assert_allclose(u[:, 1], norm_r["minuv"], atol=5e-6)
    sf = SF.read_table(rd / "slfeng.tt")
    assert len(sf) == orc_r.esmax
    np.testing.assert_allclose(sf[:, 1], norm_r["eself"], rtol=1e-14, atol=1e-300)
    av = SF.read_table(sd / "aveuv.tt")
    assert av.shape == (1, 1 + orc_s.numslv)
    np.testing.assert_allclose(av[0, 1:], norm_s["slnuv"], atol=5e-6)


def test_slvfe_from_files_matches_arrays(engine_lib, oracle_mod, tmp_path):
    """erdst's files -> slvfe gives the delta mu of the in-memory distributions."""
    (orc_s, norm_s, _, mesh_s, sd), (orc_r, norm_r, _, mesh_r, rd) = _soln_and_refs(oracle_mod, tmp_path)
    _, middle, _, spec = SF.representative_bins(mesh_s["uvcrd"], mesh_s["uvmax"], mesh_s["uvsoft"])
    a = SF.delta_mu(norm_s["edens"], norm_r["edens"], norm_r["ecorr"], middle, spec, 300.0,
                    [float(norm_s["slnuv"][0])])
    b = SF.delta_mu_from_files(sd, rd, 300.0)
    assert np.isfinite(b[1])
    # g15.7 bin middles and f15.5 aveuv carry ~1e-7 relative and 5e-6 absolute
    assert b[1] == pytest.approx(a[1], abs=2e-5)


def test_engstore_divisions(engine_lib, oracle_mod, tmp_path):
    w = S.make_workload(2, small=True, maxins=16)
    prm = dict(w.params, corrcal=1, selfcal=1)
    _, norm, av, mesh = _oracle_division(oracle_mod, w, prm, w.topo, 1)
    avediv = np.vstack([av, av * 1.5, av * 2.0])
    for d in (1, 2, 3):
        IO.write_engstore(tmp_path, prm, mesh, norm, d, 3, avediv[:d].tolist() + [[0, 0]] * (3 - d))
    names = sorted(os.listdir(tmp_path))
    assert names == ["corref.01", "corref.02", "corref.03", "engref.01", "engref.02", "engref.03",
                     "slfeng.01", "slfeng.02", "slfeng.03", "uvrange.tt", "weight_refs"]
    t = SF.read_table(tmp_path / "weight_refs")
    np.testing.assert_allclose(t[:, 0], [1, 2, 3])
    np.testing.assert_allclose(t[:, 1], avediv[:, 0], rtol=5.01e-8)
    with pytest.raises(IO.IOError_, match="sto_div"):
        IO.write_engstore(tmp_path, prm, mesh, norm, 4, 3, avediv)
    with pytest.raises(IO.IOError_, match="sto_opn"):
        IO.write_engstore(tmp_path / "no" / "such" / "dir", prm, mesh, norm, 1, 3, avediv)


def _vmdfio_cell(box):
    """vmdfio.c:355-373 on the plugin's FP32 A, B, C, alpha, beta, gamma."""
    A_, B, Cc, al, be, ga = (float(v) for v in box)
    x, y = np.cos(ga * np.pi / 180.0), np.sin(ga * np.pi / 180.0)
    u = np.cos(be * np.pi / 180.0)
    v = (np.cos(al * np.pi / 180.0) - x * u) / y
    w = np.sqrt(1.0 - u * u - v * v)
    return np.array([A_, 0, 0, B * x, B * y, 0, Cc * u, Cc * v, Cc * w], dtype=np.float32)


@pytest.mark.parametrize("variant", ["charmm_cos_le", "charmm_cos_be", "namd_deg", "xplor", "triclinic", "dim4"])
def test_dcd_reader_matches_reference_plugin(engine_lib, oracle_mod, tmp_path, variant):
    """The library's reader against the reference's own DCD reader (its vendored VMD plugin,
    built from source by the oracle recipe): the same coordinates, and the cell vmdfio builds."""
    fr = _frames(3, natoms=11, seed=4)
    par = (40.0, 42.0, 45.0, 70.0, 80.0, 100.0) if variant == "triclinic" else (31.0, 32.5, 33.0, 90.0, 90.0, 90.0)
    kw = dict(cells=[cell_record(*par, cosines=variant != "namd_deg")] * 3)
    if variant == "charmm_cos_be":
        kw["end"] = ">"
    if variant == "xplor":
        kw = dict(cells=None, charmm=False)
    if variant == "dim4":
        kw["dim4"] = True
    p = tmp_path / f"{variant}.dcd"
    write_dcd(p, fr, **kw)
    ref = oracle_mod.ref_dcd_frames(str(p))
    if ref is None:
        pytest.skip("the reference sources are not here to build its DCD reader")
    with IO.Trajectory(p) as t:
        ours = [t.read() for _ in range(len(ref) + 1)]
    assert len(ref) == 3 and ours[-1] is None
    for (crd, box), (c2, cell) in zip(ref, ours[:-1]):
        np.testing.assert_array_equal(c2, crd)
        if variant != "xplor":
            np.testing.assert_allclose(cell, _vmdfio_cell(box), rtol=1e-6, atol=1e-5)
