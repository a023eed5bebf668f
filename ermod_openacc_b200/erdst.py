"""erdst's trajectory loop over the library: HISTORY in, engstore's files out.

`run` follows trjmain (enganal.F90:60-105) for one process:
  * frames_per_div = maxcnf / skpcnf / engdiv (halt 'eng_par' when zero);
  * per division: engclear, then for every frame getconf_parallel
    (setconf.F90:849-986) reads skpcnf configurations from HISTORY, keeping
    the last with its SysWght weight and the MolPrm-style permutation, and
    engconst runs on it;
  * flexible solutes (slttype 3) read one SltConf conformation per insertion
    with its SltWght weight and the insstructure RMSD filter (getsolute,
    insertion.F90:393-543), wrapping around at the end of either file;
  * engstore normalises and writes the division's files (engproc.F90:630-722).
With a torch.distributed process group the frames are shared as
getconf_parallel shares them among MPI ranks (setconf.F90:931-980): each batch
of world-size frames gives rank r its r-th frame, numbered stnum + r + 1; the
SltConf conformations go to the ranks in turn, per insertion, as getsolute
hands them out (insertion.F90:458-528); engstore reduces over the ranks
(ermod_openacc_b200.parallel) and rank 0 writes the files.  The namelist
parsing stays outside: the caller passes &ene_param as a dict and the topology
objects of `ermod_openacc_b200.systems`.
"""
from __future__ import annotations

import os

import numpy as np

from . import _capi as A
from . import erdst_io as IO

__all__ = ["run", "INSSTR_NOREJECT", "INSSTR_RMSD"]

INSSTR_NOREJECT, INSSTR_RMSD = 0, 1   # insstructure (engmain.F90)


class _WeightFile:
    """'index weight' lines read in sequence (read_weight, setconf.F90:988-1013; the
    SltWght reader of getsolute wraps around at the end, insertion.F90:470-481)."""

    def __init__(self, path: str, wrap: bool):
        self.rows = []
        with open(path) as f:
            for line in f:
                t = line.split()
                if len(t) >= 2:
                    self.rows.append(float(t[1]))
        self.wrap = wrap
        self.i = 0
        if not self.rows:
            raise IO.IOError_(A.ERR_FORMAT, "wgt_frm")

    def next(self) -> float:
        if self.i >= len(self.rows):
            if not self.wrap:
                raise IO.IOError_(A.ERR_FORMAT, "wgt_len")
            self.i = 0
        v = self.rows[self.i]
        self.i += 1
        return v


class _SoluteSource:
    """getsolute (insertion.F90:393-543) with consecutive_read off: one conformation
    per insertion, the structure weight, and the RMSD filter against RefInfo's solute."""

    def __init__(self, sltconf, nsite, sltwgt=None, insstructure=INSSTR_NOREJECT, lwstr=0.0, upstr=0.0,
                 refslt=None):
        self.traj = IO.Trajectory(sltconf)
        if self.traj.natoms != nsite:
            raise IO.IOError_(A.ERR_FORMAT, "ins_siz")
        self.nsite = nsite
        self.wgt = _WeightFile(sltwgt, wrap=True) if sltwgt else None
        self.insstructure = insstructure
        self.lwstr, self.upstr = float(lwstr), float(upstr)
        if insstructure == INSSTR_RMSD:
            if refslt is None:
                raise IO.IOError_(A.ERMOD_ERR_ARG, "ins_ref")
            self.ref_crd = A.as_f32(refslt[0]).reshape(-1, 3)
            self.ref_w = A.as_f32(refslt[1]).ravel()
            if len(self.ref_w) != nsite:
                raise IO.IOError_(A.ERMOD_ERR_ARG, "ins_siz")
        self.wraps = 0   # wrap-arounds since the last accepted conformation

    def _next_conf(self):
        fr = self.traj.read()
        if fr is None:   # OUTconfig's wrap-around (setconf.F90:106-116)
            self.traj.rewind()
            self.wraps += 1
            fr = self.traj.read()
            if fr is None:
                raise IO.IOError_(A.ERR_FORMAT, "slt_trj")
        return fr[0].reshape(-1, 3)

    def next(self):
        while True:
            crd = self._next_conf()
            w = self.wgt.next() if self.wgt else 1.0
            if self.insstructure == INSSTR_NOREJECT:
                return crd, w
            r = IO.rmsd_bestfit(self.ref_crd, crd, self.ref_w)
            if self.lwstr <= r <= self.upstr:
                self.wraps = 0
                return crd, w
            if self.wraps >= 2:
                # two whole passes over SltConf without an accepted structure: the reference's
                # reading loop would never end (insertion.F90:464-506)
                raise IO.IOError_(A.ERMOD_ERR_ARG, "ins_str")

    def batch(self, n):
        conf = np.zeros((n, self.nsite, 3), dtype=np.float32)
        wgt = np.zeros(n, dtype=np.float32)
        for i in range(n):
            conf[i], wgt[i] = self.next()
        return conf, wgt

    def close(self):
        self.traj.close()


def run(params: dict, topo, hist: dict | None, history, outdir, maxcnf: int, skpcnf: int = 1, engdiv: int = 1,
        syswgt=None, permutation=None, sltconf=None, sltwgt=None, insstructure: int = INSSTR_NOREJECT,
        lwstr: float = 0.0, upstr: float = 0.0, refslt=None, engine=None, device: int = 0, dist_group=None,
        reduce_device=None) -> dict:
    """One erdst run over the HISTORY trajectory `history`, writing engstore's files into
    `outdir`.  permutation: 1-based target index of each HISTORY atom (the permutation file
    of getconf_parallel); syswgt / sltwgt: weight files; sltconf: the SltConf trajectory of
    a flexible solute; refslt: (coordinates, weights) of RefInfo's solute for insstructure 1.
    `engine` is a ready context with engclear / engconst / engstore / accum (an `Engine` is
    made on `device` when None).  dist_group: a torch.distributed group to share the frames
    over (None: this process alone); reduce_device: where the cross-rank sums run ("cuda:N"
    for NCCL, None for gloo on the host).  Returns avediv, aveuv and the frames this rank
    processed."""
    world, rank = 1, 0
    if dist_group is not None:
        import torch.distributed as dist
        world, rank = dist.get_world_size(dist_group), dist.get_rank(dist_group)
    frames_per_div = maxcnf // skpcnf // engdiv if skpcnf > 0 and engdiv > 0 else 0
    if frames_per_div <= 0:
        raise IO.IOError_(A.ERMOD_ERR_ARG, "eng_par")
    if engdiv > 99:
        raise IO.IOError_(A.ERMOD_ERR_ARG, "sto_div")
    os.makedirs(outdir, exist_ok=True)
    if engine is None:
        from .engine import Engine
        engine = Engine(params, topo, hist, device=device)
    phys = (topo.sluvid == A.PT_SOLVENT) | (topo.sluvid == A.PT_SOLUTE)
    natoms = int(np.asarray(topo.numsite)[phys].sum())
    perm = None
    if permutation is not None:
        perm = np.asarray(permutation, dtype=np.int64) - 1
        if len(perm) != natoms or np.any(np.sort(perm) != np.arange(natoms)):
            raise IO.IOError_(A.ERMOD_ERR_ARG, "set_pmt")
    soln = params["slttype"] == A.SLT_SOLN
    flex = params["slttype"] == A.SLT_REFS_FLEX
    traj = IO.Trajectory(history)
    if traj.natoms != natoms:
        traj.close()
        raise IO.IOError_(A.ERR_FORMAT, "set_trj")
    if flex and sltconf is None:
        traj.close()
        raise IO.IOError_(A.ERMOD_ERR_ARG, "ins_trj")
    wsys = _WeightFile(syswgt, wrap=False) if syswgt else None
    src = _SoluteSource(sltconf, int(topo.numsite[-1]), sltwgt, insstructure, lwstr, upstr, refslt) if flex else None
    mesh = dict(uvcrd=engine.uvcrd, uvmax=engine.uvmax, uvsoft=engine.uvsoft, escrd=engine.escrd)
    avediv = np.zeros((engdiv, 2))
    aveuv = np.zeros((engdiv, topo.numslv), dtype=np.float32) if soln else None
    stnum = 0
    processed = 0
    try:
        for div in range(1, engdiv + 1):
            engine.engclear()
            done = 0
            while done < frames_per_div:
                nread = min(world, frames_per_div - done)   # getconf_parallel's batch
                mine = None
                for iproc in range(nread):
                    pos = cell = None
                    weight = 1.0
                    for _ in range(skpcnf):
                        fr = traj.read()
                        if fr is None:
                            raise IO.IOError_(A.ERR_FORMAT, "set_trj")
                        pos, cell = fr
                        weight = wsys.next() if wsys else 1.0
                    if iproc == rank:
                        mine = (pos, cell, weight)
                if perm is not None and mine is not None:
                    p3 = mine[0].reshape(-1, 3)
                    out = np.empty_like(p3)
                    out[perm] = p3
                    mine = (out.ravel(), mine[1], mine[2])
                kw = {}
                if flex:
                    # getsolute: per insertion, one conformation for each active rank in turn
                    nins = params["maxins"]
                    confs, wgts = src.batch(nins * nread)
                    sel = np.arange(nins) * nread + rank
                    if rank < nread:
                        kw = dict(ins_conf=confs[sel].ravel(), ins_weight=wgts[sel])
                if rank < nread:
                    rc = engine.engconst(stnum + rank + 1, mine[0], mine[1], mine[2], **kw)
                    if rc < 0:
                        raise IO.IOError_(rc, "eng_cns")
                    processed += 1
                stnum += nread
                done += nread
            if world > 1:
                from . import parallel
                norm, av = parallel.engstore_all(engine, group=dist_group, device=reduce_device)
            else:
                norm, av = engine.engstore()
            avediv[div - 1] = av
            if soln:
                aveuv[div - 1] = norm["slnuv"]
            if rank == 0:
                IO.write_engstore(outdir, params, mesh, norm, div, engdiv, avediv, aveuv)
    finally:
        traj.close()
        if src is not None:
            src.close()
    return dict(avediv=avediv, aveuv=aveuv, frames=processed)
