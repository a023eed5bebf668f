"""Python host mirror of erdst's engproc interface over the C-ABI.

`Engine.engclear / engconst / engstore` follow the reference's
engclear (erdst/engproc.F90:321-340), engconst(stnum) (:353-517) and
engstore(stnum) (:520-725).  Errors the reference raises through
halt_with_error come back as `ErmodError` carrying the same 7-character
code; the `mbin` warning is returned as the positive status
ERMOD_WARN_MBIN so the caller can apply the reference's
force_calculation policy (erdst/mpiproc.F90:238-252).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _capi as A
from . import systems as S


class ErmodError(RuntimeError):
    def __init__(self, code: int, name: str):
        super().__init__(f"{name} ({code})")
        self.code = code
        self.name = name


def enginit_mesh(hist: dict | None, numslv: int):
    """enginit's energy mesh (engproc.F90:171-281) through the library."""
    lib = A.load_library()
    h = S.hist_struct(hist)
    ermax, esmax = C.c_int32(), C.c_int32()
    rc = lib.ermod_enginit_mesh(C.byref(h), numslv, None, None, None, None, C.byref(ermax), C.byref(esmax))
    if rc != 0:
        raise ErmodError(rc, "eng_ecd")
    uvcrd = np.zeros(ermax.value)
    uvmax = np.zeros(numslv, dtype=np.int32)
    uvsoft = np.zeros(numslv, dtype=np.int32)
    escrd = np.zeros(esmax.value)
    lib.ermod_enginit_mesh(C.byref(h), numslv, A.ptr(uvcrd, C.c_double), A.ptr(uvmax, C.c_int32),
                           A.ptr(uvsoft, C.c_int32), A.ptr(escrd, C.c_double), C.byref(ermax), C.byref(esmax))
    return uvcrd, uvmax, uvsoft, escrd


class Engine:
    """One engine context on one GPU."""

    def __init__(self, params: dict, topo: S.Topology, hist: dict | None = None, device: int = 0):
        self.lib = A.load_library()
        self.params = dict(params)
        self.topo = topo
        self.uvcrd, self.uvmax, self.uvsoft, self.escrd = enginit_mesh(hist, topo.numslv)
        self.ermax, self.esmax, self.numslv = len(self.uvcrd), len(self.escrd), topo.numslv
        self._ps = S.params_struct(self.params)
        self._ts, self._keep = topo.as_struct()
        self._ms = A.ErmodMesh(numslv=self.numslv, ermax=self.ermax, esmax=self.esmax,
                               uvcrd=A.ptr(self.uvcrd, C.c_double), uvmax=A.ptr(self.uvmax, C.c_int32),
                               uvsoft=A.ptr(self.uvsoft, C.c_int32), escrd=A.ptr(self.escrd, C.c_double))
        self.ctx = C.c_void_p()
        rc = self.lib.ermod_create(C.byref(self.ctx), device, C.byref(self._ps), C.byref(self._ts), C.byref(self._ms))
        if rc != 0:
            name = self.lib.ermod_last_error(self.ctx).decode() if self.ctx else "create"
            self.close()
            raise ErmodError(rc, name)
        sl, md, ns, na = C.c_int32(), C.c_int32(), C.c_int32(), C.c_int32()
        self.lib.ermod_get_sizes(self.ctx, C.byref(sl), C.byref(md), C.byref(ns), C.byref(na))
        self.slvmax, self.maxdst, self.nsite_slt, self.natoms = sl.value, md.value, ns.value, na.value

    def close(self):
        if getattr(self, "ctx", None):
            self.lib.ermod_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        self.close()

    def _check(self, rc: int) -> int:
        if rc < 0:
            raise ErmodError(rc, self.lib.ermod_last_error(self.ctx).decode())
        return rc

    def last_error(self) -> str:
        return self.lib.ermod_last_error(self.ctx).decode()

    def engclear(self):
        return self._check(self.lib.ermod_engclear(self.ctx))

    def engconst(self, stnum: int, sitepos, cell, stat_weight_system: float = 1.0, ins_conf=None,
                 ins_weight=None) -> int:
        sp = A.as_f32(sitepos)
        cl = A.as_f32(cell)
        ic = None if ins_conf is None else A.as_f32(ins_conf)
        iw = None if ins_weight is None else A.as_f32(ins_weight)
        fl = np.zeros(max(1, self.maxdst * self.numslv), dtype=np.float32)
        rc = self.lib.ermod_engconst(self.ctx, stnum, A.ptr(sp, C.c_float), A.ptr(cl, C.c_float),
                                     stat_weight_system, A.ptr(ic, C.c_float), A.ptr(iw, C.c_float),
                                     A.ptr(fl, C.c_float))
        self.flceng = fl.reshape(self.maxdst, self.numslv) if self.numslv else fl
        return self._check(rc)

    def engconst_dev(self, stnum: int, sitepos_ptr: int, cell, stat_weight_system: float = 1.0,
                     ins_conf_ptr: int | None = None, ins_weight_ptr: int | None = None) -> int:
        cl = A.as_f32(cell)
        rc = self.lib.ermod_engconst_dev(self.ctx, stnum, C.c_void_p(sitepos_ptr), A.ptr(cl, C.c_float),
                                         stat_weight_system, C.c_void_p(ins_conf_ptr) if ins_conf_ptr else None,
                                         C.c_void_p(ins_weight_ptr) if ins_weight_ptr else None)
        return self._check(rc)

    def _accum_struct(self, ecorr: bool = True):
        ed = np.zeros(self.ermax)
        ec = np.zeros(self.ermax * self.ermax) if self.params["corrcal"] and ecorr else None
        es = np.zeros(self.esmax) if self.params["selfcal"] else None
        sl = np.zeros(self.numslv, dtype=np.float32)
        mn = np.zeros(self.numslv + 1, dtype=np.float32)
        mx = np.zeros(self.numslv + 1, dtype=np.float32)
        acc = A.ErmodAccum(edens=A.ptr(ed, C.c_double), ecorr=A.ptr(ec, C.c_double), eself=A.ptr(es, C.c_double),
                           slnuv=A.ptr(sl, C.c_float), minuv=A.ptr(mn, C.c_float), maxuv=A.ptr(mx, C.c_float))
        return acc, (ed, ec, es, sl, mn, mx)

    def _accum_dict(self, acc, arrs):
        ed, ec, es, sl, mn, mx = arrs
        return dict(edens=ed, ecorr=None if ec is None else ec.reshape(self.ermax, self.ermax), eself=es, slnuv=sl,
                    minuv=mn, maxuv=mx, avslf=acc.avslf, engnorm=acc.engnorm, engsmpl=acc.engsmpl,
                    voffset=acc.voffset, voffset_initialized=acc.voffset_initialized)

    def set_refstructure(self, refspec: int, host_crd, host_w, slt_crd, slt_w) -> int:
        """RefInfo reference structure for insposition 5 / 6 (load_refstructure,
        insertion.F90:676-770): the atoms of the refspec species (bit mask over uvspec) in
        molecule order and the solute, with their fit weights."""
        hc, hw, sc, sw = (A.as_f32(x) for x in (host_crd, host_w, slt_crd, slt_w))
        self._ref = (hc, hw, sc, sw)
        return self._check(self.lib.ermod_set_refstructure(self.ctx, int(refspec), len(hw), A.ptr(hc, C.c_float),
                                                           A.ptr(hw, C.c_float), A.ptr(sc, C.c_float),
                                                           A.ptr(sw, C.c_float)))

    def accum(self, ecorr: bool = True) -> dict:
        """Raw accumulators of the current division (engstore's inputs); ecorr=False leaves
        the ermax^2 correlation matrix on the device (its entry is None)."""
        acc, arrs = self._accum_struct(ecorr)
        self._check(self.lib.ermod_fetch_accum(self.ctx, C.byref(acc)))
        return self._accum_dict(acc, arrs)

    def engstore(self):
        """engstore's normalisation (engproc.F90:609-628): (normalised dict, avediv[2])."""
        acc, arrs = self._accum_struct()
        av = np.zeros(2)
        self._check(self.lib.ermod_engstore(self.ctx, C.byref(acc), A.ptr(av, C.c_double)))
        return self._accum_dict(acc, arrs), av

    def uvengy(self):
        """(uvengy[maxdst, slvmax], uvengy0[maxdst]) of the last frame (needs keep_uvengy=1)."""
        u = np.zeros(self.maxdst * self.slvmax)
        u0 = np.zeros(self.maxdst)
        self._check(self.lib.ermod_get_uvengy(self.ctx, A.ptr(u, C.c_double), A.ptr(u0, C.c_double)))
        return u.reshape(self.maxdst, self.slvmax), u0

    def uvengy0(self):
        u0 = np.zeros(self.maxdst)
        self._check(self.lib.ermod_get_uvengy(self.ctx, None, A.ptr(u0, C.c_double)))
        return u0

    def insertions(self):
        o = np.zeros(3 * self.nsite_slt * self.maxdst, dtype=np.float32)
        w = np.zeros(self.maxdst)
        self._check(self.lib.ermod_get_insertions(self.ctx, A.ptr(o, C.c_float), A.ptr(w, C.c_double)))
        return o, w

    STAGES = ["total", "prepare", "insert", "real", "spread", "r2c", "influence", "c2r", "gather", "bin",
              "weights_edens", "ecorr", "chunks", "transpose", "pme_plane", "pme_rows", "site_tables"]

    def timings(self):
        """Device milliseconds per stage of the last engconst (CUDA events on the engine stream)."""
        t = np.zeros(len(self.STAGES), dtype=np.float32)
        self.lib.ermod_get_timings(self.ctx, A.ptr(t, C.c_float), len(self.STAGES))
        return dict(zip(self.STAGES, t.tolist()))

    def launch_count(self) -> int:
        return int(self.lib.ermod_get_launch_count(self.ctx))

    def last_ms(self) -> float:
        """Device time of the last frame (the stage timings' total)."""
        return self.timings()["total"]

    def proposal_config(self, voxels_per_side: int, mix_uniform: float = 0.1, params=None, feature_cells: int = 0):
        """Voxel grid (and feature-cell grid, 0: twice as fine) of the insertion proposal; with `params`
        (FP32 network parameters) and params['proposal'] == PROPOSAL_LEARNED, insertions are drawn from
        the network's proposal."""
        pp = None if params is None else np.ascontiguousarray(params, dtype=np.float32)
        self._check(self.lib.ermod_proposal_config(self.ctx, voxels_per_side, feature_cells, mix_uniform,
                                                   A.ptr(pp, C.c_float)))

    def insertion_samples(self):
        """(features [maxdst, 64], total solute-solvent energy [maxdst], voxel [maxdst]) of the last frame."""
        f = np.zeros(self.maxdst * 64, dtype=np.float32)
        e = np.zeros(self.maxdst)
        v = np.zeros(self.maxdst, dtype=np.int32)
        self._check(self.lib.ermod_get_insertion_samples(self.ctx, A.ptr(f, C.c_float), A.ptr(e, C.c_double),
                                                         A.ptr(v, C.c_int32)))
        return f.reshape(self.maxdst, 64), e, v

    def paths(self) -> dict:
        """Resolved kernel choices: spectrum_path 1 cuFFT / 2 fused direct / 3 fused spread, ecorr_path."""
        sp, ep = C.c_int32(), C.c_int32()
        self._check(self.lib.ermod_get_paths(self.ctx, C.byref(sp), C.byref(ep)))
        return dict(spectrum_path=sp.value, ecorr_path=ep.value)


class Batch:
    """Solutes sharing one solvent frame, run as one CUDA-graph launch per frame
    (ermod_batch_*).  Each member Engine keeps its own accumulators, bit-identical
    to running it alone."""

    def __init__(self, members: list[Engine]):
        self.lib = A.load_library()
        self.members = list(members)
        arr = (C.c_void_p * len(self.members))(*[m.ctx.value for m in self.members])
        self.h = C.c_void_p()
        rc = self.lib.ermod_batch_create(C.byref(self.h), len(self.members), arr)
        if rc != 0:
            raise ErmodError(rc, "batch")

    def close(self):
        if getattr(self, "h", None):
            self.lib.ermod_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def engconst(self, stnum: int, sitepos, cell, stat_weight_system: float = 1.0) -> int:
        sp, cl = A.as_f32(sitepos), A.as_f32(cell)
        rc = self.lib.ermod_batch_engconst(self.h, stnum, A.ptr(sp, C.c_float), A.ptr(cl, C.c_float),
                                           stat_weight_system)
        if rc < 0:
            raise ErmodError(rc, self.lib.ermod_batch_last_error(self.h).decode())
        return rc

    def engconst_dev(self, stnum: int, sitepos_ptr: int, cell, stat_weight_system: float = 1.0) -> int:
        cl = A.as_f32(cell)
        rc = self.lib.ermod_batch_engconst_dev(self.h, stnum, C.c_void_p(sitepos_ptr), A.ptr(cl, C.c_float),
                                               stat_weight_system)
        if rc < 0:
            raise ErmodError(rc, self.lib.ermod_batch_last_error(self.h).decode())
        return rc

    def last_ms(self) -> float:
        return float(self.lib.ermod_batch_last_ms(self.h))
