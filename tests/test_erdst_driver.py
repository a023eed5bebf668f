"""The erdst trajectory loop (ermod_openacc_b200.erdst.run): HISTORY / SysWght /
SltConf / SltWght in, engstore's files out.  CPU tests drive it with the oracle behind
the engine interface; the GPU test compares the CUDA engine's files with those."""
import os

import numpy as np
import pytest

from ermod_openacc_b200 import _capi as A
from ermod_openacc_b200 import erdst
from ermod_openacc_b200 import erdst_io as IO
from ermod_openacc_b200 import slvfe as SF
from ermod_openacc_b200 import systems as S
from _dcd import write_dcd


class OracleEngine:
    """The oracle behind the engine interface the loop drives (test infrastructure)."""

    def __init__(self, oracle_mod, params, topo, hist):
        self.o = oracle_mod.Oracle(params, topo, hist, precision=8)
        self.params = params
        self.uvcrd, self.uvmax, self.uvsoft, self.escrd = self.o.uvcrd, self.o.uvmax, self.o.uvsoft, self.o.escrd
        self.calls = []

    def engclear(self):
        self.o.engclear()

    def engconst(self, stnum, pos, cell, w=1.0, ins_conf=None, ins_weight=None):
        self.calls.append(dict(stnum=stnum, pos=pos.copy(), cell=cell.copy(), w=w,
                               ins_conf=None if ins_conf is None else ins_conf.copy(),
                               ins_weight=None if ins_weight is None else ins_weight.copy()))
        return self.o.engconst(stnum, pos, cell, w, ins_conf=ins_conf, ins_weight=ins_weight)

    def accum(self):
        return self.o.accum()

    def engstore(self):
        raw = self.o.accum()
        norm = self.o.accum(normalise=True)
        sgn = -1.0 if self.params["slttype"] == A.SLT_SOLN else 1.0
        with np.errstate(divide="ignore"):
            av = np.array([raw["engnorm"] / raw["engsmpl"], raw["voffset"] + sgn * self.params["temp"] *
                           np.log(norm["avslf"])])
        return norm, av


def _history(tmp_path, w, nframes, perm=None, name="HISTORY.dcd"):
    frames, cells = [], []
    for k in range(nframes):
        pos, cell = w.frame(k)
        p3 = np.asarray(pos, dtype=np.float32).reshape(-1, 3)
        if perm is not None:   # HISTORY atom i is program atom perm[i]
            p3 = p3[perm]
        frames.append(p3)
        c = np.asarray(cell, dtype=np.float64).reshape(3, 3, order="F")
        cells.append([c[0, 0], 0.0, c[1, 1], 0.0, 0.0, c[2, 2]])   # orthorhombic: cosines 0
    path = tmp_path / name
    write_dcd(path, frames, cells)
    return path


def _read_frames(path, n):
    with IO.Trajectory(path) as t:
        return [t.read() for _ in range(n)]


def _expected(oracle_mod, prm, topo, hist, frames, weights, stnums):
    eng = OracleEngine(oracle_mod, prm, topo, hist)
    for (pos, cell), wv, st in zip(frames, weights, stnums):
        assert eng.engconst(st, pos, cell, wv) >= 0
    return eng.engstore()


def test_refs_divisions_weights_and_skips(engine_lib, oracle_mod, tmp_path):
    w = S.make_workload(2, small=True, maxins=48)
    prm = dict(w.params, selfcal=1)
    hist_path = _history(tmp_path, w, 8)
    wfile = tmp_path / "SysWght"
    wts = [1.0, 0.5, 2.0, 1.5, 0.75, 1.25, 3.0, 0.25]
    wfile.write_text("".join(f"{i + 1} {v}\n" for i, v in enumerate(wts)))
    out = tmp_path / "out"
    eng = OracleEngine(oracle_mod, prm, w.topo, w.hist)
    res = erdst.run(prm, w.topo, w.hist, hist_path, out, maxcnf=8, skpcnf=2, engdiv=2, syswgt=wfile, engine=eng)
    assert res["frames"] == 4
    # skpcnf 2: frames 2, 4 | 6, 8 with their own weights, numbered 1..4
    assert [c["stnum"] for c in eng.calls] == [1, 2, 3, 4]
    assert [c["w"] for c in eng.calls] == [wts[1], wts[3], wts[5], wts[7]]
    fr = _read_frames(hist_path, 8)
    for c, k in zip(eng.calls, (1, 3, 5, 7)):
        np.testing.assert_array_equal(c["pos"], fr[k][0])
    assert sorted(os.listdir(out)) == ["corref.01", "corref.02", "engref.01", "engref.02", "slfeng.01",
                                       "slfeng.02", "uvrange.tt", "weight_refs"]
    for div, ks, st in ((1, (1, 3), (1, 2)), (2, (5, 7), (3, 4))):
        norm, av = _expected(oracle_mod, prm, w.topo, w.hist, [fr[k] for k in ks], [wts[k] for k in ks], st)
        e = SF.read_engfile(out / f"engref.{div:02d}")
        np.testing.assert_allclose(e["ratio"], norm["edens"], rtol=1e-13, atol=1e-300)
        # division 2 keeps the run's first voffset, the fresh oracle its own: rounding only
        np.testing.assert_allclose(SF.read_corfile(out / f"corref.{div:02d}", len(e["ratio"])), norm["ecorr"].T,
                                   rtol=1e-13, atol=1e-300)
        # engnorm / engsmpl carries exp(voffset / kT) of the run's first frame: exact for
        # division 1; the voffset-free second column in both
        if div == 1:
            np.testing.assert_allclose(res["avediv"][0], av, rtol=1e-12)
        assert res["avediv"][div - 1, 1] == pytest.approx(av[1], rel=1e-10, abs=1e-12)
    t = SF.read_table(out / "weight_refs")
    np.testing.assert_allclose(t[:, 1], res["avediv"][:, 0], rtol=5.01e-8)


def test_permutation(engine_lib, oracle_mod, tmp_path):
    w = S.make_workload(2, small=True, maxins=24)
    n = int(np.asarray(w.topo.numsite)[(w.topo.sluvid == A.PT_SOLVENT) | (w.topo.sluvid == A.PT_SOLUTE)].sum())
    rng = np.random.default_rng(2)
    perm = rng.permutation(n)                   # HISTORY atom i is program atom perm[i]
    plain = _history(tmp_path, w, 2, name="plain.dcd")
    shuffled = _history(tmp_path, w, 2, perm=perm, name="perm.dcd")
    e1 = OracleEngine(oracle_mod, w.params, w.topo, w.hist)
    erdst.run(w.params, w.topo, w.hist, plain, tmp_path / "a", maxcnf=2, engine=e1)
    e2 = OracleEngine(oracle_mod, w.params, w.topo, w.hist)
    erdst.run(w.params, w.topo, w.hist, shuffled, tmp_path / "b", maxcnf=2, engine=e2, permutation=perm + 1)
    for c1, c2 in zip(e1.calls, e2.calls):
        np.testing.assert_array_equal(c1["pos"], c2["pos"])
    assert open(tmp_path / "a" / "engref.tt").read() == open(tmp_path / "b" / "engref.tt").read()
    with pytest.raises(IO.IOError_, match="set_pmt"):
        erdst.run(w.params, w.topo, w.hist, shuffled, tmp_path / "c", maxcnf=2, engine=e2,
                  permutation=np.ones(n, dtype=int))


def test_soln_aveuv(engine_lib, oracle_mod, tmp_path):
    w = S.make_workload(1, small=True)
    hist_path = _history(tmp_path, w, 4)
    eng = OracleEngine(oracle_mod, w.params, w.topo, w.hist)
    res = erdst.run(w.params, w.topo, w.hist, hist_path, tmp_path / "o", maxcnf=4, engdiv=2, engine=eng)
    av = SF.read_table(tmp_path / "o" / "aveuv.tt")
    assert av.shape == (2, 1 + w.topo.numslv)
    np.testing.assert_allclose(av[:, 1:], res["aveuv"], atol=5e-6)
    assert os.path.exists(tmp_path / "o" / "engsln.01") and os.path.exists(tmp_path / "o" / "engsln.02")


def _flex_setup(tmp_path, nconf=7):
    w = S.make_workload(2, small=True, maxins=5)
    kinds = [A.PT_TEST_FLEX if k == A.PT_TEST_RIGID else k for k in w.topo.kinds]
    topo = S.Topology(w.topo.species, w.topo.counts, kinds)
    prm = dict(w.params, slttype=A.SLT_REFS_FLEX)
    ref = np.asarray(w.topo.bfcoord, dtype=np.float64).reshape(-1, 3)
    rng = np.random.default_rng(9)
    confs = [ref + rng.normal(scale=s, size=ref.shape) for s in np.linspace(0.0, 0.6, nconf)]
    write_dcd(tmp_path / "SltConf.dcd", confs, None, charmm=False)
    (tmp_path / "SltWght").write_text("".join(f"{i + 1} {1.0 + 0.1 * i}\n" for i in range(nconf)))
    return w, topo, prm, ref, confs


def test_flexible_solute_conformations_weights_and_rmsd_filter(engine_lib, oracle_mod, tmp_path):
    w, topo, prm, ref, confs = _flex_setup(tmp_path)
    hist_path = _history(tmp_path, w, 3)
    wts = np.ones(len(ref), dtype=np.float32)
    rms = np.array([IO.rmsd_bestfit(ref, c, wts) for c in confs])
    lw, up = 0.05, 0.6
    ok = np.nonzero((rms >= lw) & (rms <= up))[0]
    assert 1 < len(ok) < len(confs)
    eng = OracleEngine(oracle_mod, prm, topo, w.hist)
    erdst.run(prm, topo, w.hist, hist_path, tmp_path / "o", maxcnf=3, engine=eng,
              sltconf=tmp_path / "SltConf.dcd", sltwgt=tmp_path / "SltWght",
              insstructure=erdst.INSSTR_RMSD, lwstr=lw, upstr=up, refslt=(ref, wts))
    # accepted conformations in file order, wrapping around, with their own weights
    seq = [ok[i % len(ok)] for i in range(3 * prm["maxins"])]
    got_c = np.concatenate([c["ins_conf"].reshape(-1, len(ref), 3) for c in eng.calls])
    got_w = np.concatenate([c["ins_weight"] for c in eng.calls])
    for g, k in zip(got_c, seq):
        np.testing.assert_array_equal(g, np.asarray(confs[k], dtype=np.float32))
    np.testing.assert_allclose(got_w, [1.0 + 0.1 * k for k in seq], rtol=1e-6)
    # no filter: every conformation in order
    eng2 = OracleEngine(oracle_mod, prm, topo, w.hist)
    erdst.run(prm, topo, w.hist, hist_path, tmp_path / "p", maxcnf=1, engine=eng2,
              sltconf=tmp_path / "SltConf.dcd")
    np.testing.assert_array_equal(eng2.calls[0]["ins_conf"].reshape(-1, len(ref), 3),
                                  np.asarray(confs[:5], dtype=np.float32))
    assert np.all(eng2.calls[0]["ins_weight"] == 1.0)


def test_no_accepted_structure_is_an_error(engine_lib, oracle_mod, tmp_path):
    w, topo, prm, ref, confs = _flex_setup(tmp_path)
    hist_path = _history(tmp_path, w, 1)
    eng = OracleEngine(oracle_mod, prm, topo, w.hist)
    with pytest.raises(IO.IOError_, match="ins_str"):
        erdst.run(prm, topo, w.hist, hist_path, tmp_path / "o", maxcnf=1, engine=eng,
                  sltconf=tmp_path / "SltConf.dcd", insstructure=erdst.INSSTR_RMSD, lwstr=5.0, upstr=6.0,
                  refslt=(ref, np.ones(len(ref))))


def test_run_errors(engine_lib, oracle_mod, tmp_path):
    w = S.make_workload(2, small=True, maxins=8)
    hist_path = _history(tmp_path, w, 2)
    eng = OracleEngine(oracle_mod, w.params, w.topo, w.hist)
    with pytest.raises(IO.IOError_, match="eng_par"):
        erdst.run(w.params, w.topo, w.hist, hist_path, tmp_path / "o", maxcnf=2, engdiv=3, engine=eng)
    with pytest.raises(IO.IOError_, match="set_trj"):          # fewer frames than maxcnf
        erdst.run(w.params, w.topo, w.hist, hist_path, tmp_path / "o", maxcnf=4, engine=eng)
    w1 = S.make_workload(1, small=True)
    with pytest.raises(IO.IOError_, match="set_trj"):          # atom count of another system
        erdst.run(w1.params, w1.topo, w1.hist, hist_path, tmp_path / "o", maxcnf=1,
                  engine=OracleEngine(oracle_mod, w1.params, w1.topo, w1.hist))


@pytest.mark.gpu
def test_gpu_engine_files_match_oracle(engine_lib, oracle_mod, tmp_path):
    """The CUDA engine behind the same loop writes the files the FP64 oracle writes,
    within the engine's tolerances (normalised distributions at 5e-5 relative)."""
    from ermod_openacc_b200 import Engine
    w = S.make_workload(2, small=True, maxins=64)
    hist_path = _history(tmp_path, w, 4)
    prm = dict(w.params, keep_uvengy=1)
    gpu = Engine(prm, w.topo, w.hist)
    erdst.run(prm, w.topo, w.hist, hist_path, tmp_path / "g", maxcnf=4, engdiv=2, engine=gpu)
    ins = []
    # the oracle on the GPU's placements: flexible, file-driven, unchanged
    orc_prm = dict(prm, slttype=A.SLT_REFS_FLEX, insposition=A.INSPOS_NOCHANGE, insorient=A.INSROT_NOCHANGE)
    kinds = [A.PT_TEST_FLEX if k == A.PT_TEST_RIGID else k for k in w.topo.kinds]
    topo_f = S.Topology(w.topo.species, w.topo.counts, kinds)
    gpu2 = Engine(prm, w.topo, w.hist)
    fr = _read_frames(hist_path, 4)
    for k, (pos, cell) in enumerate(fr):
        assert gpu2.engconst(k + 1, pos, cell) >= 0
        ins.append(gpu2.insertions()[0])
    orc = OracleEngine(oracle_mod, orc_prm, topo_f, w.hist)
    for div in (1, 2):
        orc.engclear()
        for k in ((0, 1) if div == 1 else (2, 3)):
            assert orc.engconst(k + 1, fr[k][0], fr[k][1], 1.0, ins_conf=ins[k].ravel()) >= 0
        norm, _ = orc.engstore()
        e = SF.read_engfile(tmp_path / "g" / f"engref.{div:02d}")
        assert e["ratio"].sum() == pytest.approx(norm["edens"].sum(), rel=5e-5)
        # bins identical except energies at a mesh edge: a few counts move to a neighbour
        assert np.abs(e["ratio"] - norm["edens"]).sum() <= 1e-3 * norm["edens"].sum()


def test_slvfe_merge_mode_over_divisions(engine_lib, oracle_mod, tmp_path):
    """erdst's division files -> slvfe's merge mode (datread / wrtmerge): per-block delta mu from
    the weight-averaged runs, the mean and the 95 % error 2 s / sqrt(n)."""
    w = S.make_workload(1, small=True)
    sd, rd = tmp_path / "soln", tmp_path / "refs"
    erdst.run(w.params, w.topo, w.hist, _history(tmp_path, w, 4, name="sln.dcd"), sd, maxcnf=4, engdiv=4,
              engine=OracleEngine(oracle_mod, w.params, w.topo, w.hist))
    topo = S.Topology([S.water(), S.lj_site()], [w.nside ** 3, 1], [A.PT_SOLVENT, A.PT_TEST_RIGID])
    prm = S.default_params(ms1max=32, maxins=500, selfcal=0)
    wr = S.Workload("refs-ljsite", prm, topo, w.hist, w.box, w.nside, 4, w.seed + 11)
    erdst.run(prm, topo, w.hist, _history(tmp_path, wr, 4, name="ref.dcd"), rd, maxcnf=4, engdiv=2,
              engine=OracleEngine(oracle_mod, prm, topo, w.hist))
    out = SF.merge_mode(sd, rd, 300.0, numdiv=2, group=3)
    assert out["numdiv"] == 2 and len(out["blocks"]) == 2
    # block 1 by hand: soln runs 1-2 weighted by weight_soln, refs runs 1-2 by weight_refs
    ws = SF.read_table(sd / "weight_soln")[:, 1]
    wrf = SF.read_table(rd / "weight_refs")[:, 1]
    wrf = wrf / wrf.sum()
    e = [SF.read_engfile(sd / f"engsln.{i:02d}") for i in (1, 2)]
    r = [SF.read_engfile(rd / f"engref.{i:02d}") for i in (1, 2)]
    n = len(e[0]["ratio"])
    chi = sum(wi * SF.read_corfile(rd / f"corref.{i:02d}", n) for wi, i in zip(wrf, (1, 2)))
    wb = ws[:2] / ws[:2].sum()
    uv = SF.read_table(sd / "aveuv.tt")[:2, 1:]
    dm = SF.delta_mu(wb[0] * e[0]["ratio"] + wb[1] * e[1]["ratio"], wrf[0] * r[0]["ratio"] + wrf[1] * r[1]["ratio"],
                     chi, e[0]["middle"], e[0]["spec"], 300.0, wb @ uv, group=3)[1]
    assert out["blocks"][0] == pytest.approx(dm, rel=1e-12, abs=1e-12)
    b = out["blocks"]
    assert out["mean"] == pytest.approx(b.mean(), rel=1e-14)
    assert out["error95"] == pytest.approx(2.0 * np.std(b, ddof=1) / np.sqrt(2), rel=1e-9)
    # numdiv that does not divide the runs moves up to the next divisor; 0 takes every run
    assert SF.merge_mode(sd, rd, 300.0, numdiv=3, group=3)["numdiv"] == 4
    assert SF.merge_mode(sd, rd, 300.0, numdiv=0, group=3)["numdiv"] == 4
    # the default scan of groups 1..5, headlined at pickgr 3
    scan = SF.merge_scan(sd, rd, 300.0, numdiv=2)
    assert sorted(scan["table"]) == [(g, 0) for g in range(1, 6)] and scan["pickgr"] == 3
    assert scan["picked"]["mean"] == pytest.approx(out["mean"], rel=1e-14)



def _dist_rank(rank, port, hist_path, outdir, engdiv):
    import os
    import torch.distributed as dist
    import oracle
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=2)
    w = S.make_workload(2, small=True, maxins=24)
    prm = dict(w.params, selfcal=1)
    eng = OracleEngine(oracle, prm, w.topo, w.hist)
    res = erdst.run(prm, w.topo, w.hist, hist_path, outdir, maxcnf=4, engdiv=engdiv, engine=eng,
                    dist_group=dist.group.WORLD)
    assert res["frames"] == 4 // 2
    # the reference's frame numbering: rank r takes frames r+1, r+3 (stnum + r + 1 per batch)
    assert [c["stnum"] for c in eng.calls] == [rank + 1, rank + 3]
    dist.barrier()
    dist.destroy_process_group()


def test_frames_shared_over_two_ranks_match_one_process(engine_lib, oracle_mod, tmp_path):
    """getconf_parallel's frame sharing and engstore's reduction on two gloo ranks (CPU): rank 0's
    files equal those of one process that ran every frame, to the rounding of the voffset rescale."""
    import socket
    import torch.multiprocessing as mp
    w = S.make_workload(2, small=True, maxins=24)
    prm = dict(w.params, selfcal=1)
    hist_path = _history(tmp_path, w, 4)
    one = OracleEngine(oracle_mod, prm, w.topo, w.hist)
    erdst.run(prm, w.topo, w.hist, hist_path, tmp_path / "one", maxcnf=4, engdiv=2, engine=one)
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    mp.spawn(_dist_rank, args=(port, hist_path, tmp_path / "two", 2), nprocs=2, join=True)
    assert sorted(os.listdir(tmp_path / "two")) == sorted(os.listdir(tmp_path / "one"))
    for div in (1, 2):
        a = SF.read_engfile(tmp_path / "one" / f"engref.{div:02d}")
        b = SF.read_engfile(tmp_path / "two" / f"engref.{div:02d}")
        np.testing.assert_allclose(b["ratio"], a["ratio"], rtol=1e-12, atol=1e-300)
        n = len(a["ratio"])
        np.testing.assert_allclose(SF.read_corfile(tmp_path / "two" / f"corref.{div:02d}", n),
                                   SF.read_corfile(tmp_path / "one" / f"corref.{div:02d}", n), rtol=1e-12,
                                   atol=1e-300)
    t1, t2 = SF.read_table(tmp_path / "one" / "weight_refs"), SF.read_table(tmp_path / "two" / "weight_refs")
    np.testing.assert_allclose(t2, t1, rtol=2e-7)


def _dist_flex_rank(rank, port, root, out):
    import os
    import torch.distributed as dist
    import oracle
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=2)
    import pathlib
    root = pathlib.Path(root)
    w, topo, prm, ref, confs = _flex_setup(root / f"r{rank}", nconf=7)
    prm = dict(prm, maxins=3)
    eng = OracleEngine(oracle, prm, topo, w.hist)
    erdst.run(prm, topo, w.hist, root / "HISTORY.dcd", root / f"o{rank}", maxcnf=4, engine=eng,
              sltconf=root / f"r{rank}" / "SltConf.dcd", sltwgt=root / f"r{rank}" / "SltWght",
              dist_group=dist.group.WORLD)
    got = np.concatenate([c["ins_conf"].reshape(-1, len(ref), 3) for c in eng.calls])
    np.save(out.format(rank), got)
    dist.barrier()
    dist.destroy_process_group()


def test_conformations_handed_out_per_insertion_over_two_ranks(engine_lib, oracle_mod, tmp_path):
    """getsolute on two ranks: per insertion, one SltConf conformation for each active rank in
    turn (insertion.F90:458-528), wrapping around at the end of the file."""
    import socket
    import torch.multiprocessing as mp
    w, topo, prm, ref, confs = _flex_setup(tmp_path, nconf=7)
    _history(tmp_path, w, 4)
    for r in (0, 1):
        (tmp_path / f"r{r}").mkdir()
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    out = str(tmp_path / "conf{}.npy")
    mp.spawn(_dist_flex_rank, args=(port, str(tmp_path), out), nprocs=2, join=True)
    seq = np.arange(12) % 7          # 2 batches x 3 insertions x 2 ranks, in file order with wrap-around
    for r in (0, 1):
        got = np.load(out.format(r))
        want = [seq[b * 6 + i * 2 + r] for b in range(2) for i in range(3)]
        np.testing.assert_array_equal(got, np.asarray([confs[k] for k in want], dtype=np.float32))
