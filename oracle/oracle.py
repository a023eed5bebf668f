"""ctypes front end of the CPU oracle -- TEST INFRASTRUCTURE, NOT PRODUCT CODE.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may
import this module, and only as the checker.  The oracle restates the
reference's algorithm (see ermod_oracle.cpp); parity is unpinned by the
reference itself (it cannot be built here and ships no golden vectors) and
is pinned by published known-answer values instead (tests/test_oracle_golden.py).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from ermod_openacc_b200 import _capi as A

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
_lib = None


REF_DCD = os.path.join(HERE, "_ref", "libref_dcd.so")


def build(force: bool = False, refsrc: str | None = None) -> str:
    """Build liboracle.so; with `refsrc` (the reference's vmdplugins directory, or the
    ERMOD_REFSRC environment variable) also the reference's own DCD reader into _ref/."""
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(
            os.path.join(HERE, "ermod_oracle.cpp")):
        subprocess.run(["make", "-C", HERE, "-s"], check=True)
    # the reference's own DCD reader behind the test shim: built only where its sources are
    refsrc = refsrc or os.environ.get("ERMOD_REFSRC")
    if refsrc and os.path.isdir(refsrc) and (force or not os.path.exists(REF_DCD)):
        subprocess.run(["make", "-C", HERE, "-s", "ref", f"REFSRC={refsrc}"], check=False, capture_output=True)
    return LIB


def ref_dcd_frames(path: str):
    """Every frame of a DCD file as the reference's vendored VMD plugin reads it: a list of
    (crd [3*natoms] float32, [A, B, C, alpha, beta, gamma] float32), or None when the
    reference reader is not built here."""
    if not os.path.exists(REF_DCD):
        return None
    L = C.CDLL(REF_DCD)
    L.ref_dcd_open.restype = C.c_void_p
    L.ref_dcd_open.argtypes = [C.c_char_p, C.POINTER(C.c_int)]
    L.ref_dcd_read.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_float), C.POINTER(C.c_float)]
    L.ref_dcd_close.argtypes = [C.c_void_p]
    na = C.c_int()
    h = L.ref_dcd_open(os.fsencode(path), C.byref(na))
    if not h:
        raise RuntimeError(f"the reference DCD reader cannot open {path}")
    frames = []
    while True:
        crd = np.zeros(3 * na.value, dtype=np.float32)
        box = np.zeros(6, dtype=np.float32)
        if L.ref_dcd_read(h, na.value, crd.ctypes.data_as(C.POINTER(C.c_float)),
                          box.ctypes.data_as(C.POINTER(C.c_float))) != 0:
            break
        frames.append((crd, box))
    L.ref_dcd_close(h)
    return frames


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(LIB)
        L.orc_philox4x32_10.argtypes = [C.POINTER(C.c_uint32)] * 3
        L.orc_spline_value.restype = C.c_double
        L.orc_spline_value.argtypes = [C.c_int, C.c_double]
        L.orc_binsearch.restype = C.c_int
        L.orc_binsearch.argtypes = [C.POINTER(C.c_double), C.c_int, C.c_double]
        L.orc_enginit_mesh.restype = C.c_int
        L.orc_enginit_mesh.argtypes = [C.POINTER(A.ErmodHist), C.c_int, C.POINTER(C.c_double),
                                       C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.POINTER(C.c_double),
                                       C.POINTER(C.c_int32), C.POINTER(C.c_int32)]
        L.orc_create.restype = C.c_void_p
        L.orc_create.argtypes = [C.POINTER(A.ErmodParams), C.POINTER(A.ErmodTopology),
                                 C.POINTER(A.ErmodMesh), C.c_int, C.c_int, C.POINTER(C.c_int)]
        L.orc_destroy.argtypes = [C.c_void_p]
        L.orc_engclear.argtypes = [C.c_void_p]
        L.orc_engconst.restype = C.c_int
        L.orc_engconst.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_float), C.POINTER(C.c_float), C.c_float,
                                   C.POINTER(C.c_float), C.POINTER(C.c_float), C.POINTER(C.c_float)]
        L.orc_fetch.argtypes = [C.c_void_p, C.POINTER(A.ErmodAccum), C.c_int]
        L.orc_get_uvengy.argtypes = [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_double)]
        L.orc_get_insertions.argtypes = [C.c_void_p, C.POINTER(C.c_float)]
        L.orc_get_engfac.argtypes = [C.c_void_p, C.POINTER(C.c_double)]
        L.orc_last_error.restype = C.c_char_p
        L.orc_last_error.argtypes = [C.c_void_p]
        L.orc_get_insw.argtypes = [C.c_void_p, C.POINTER(C.c_double)]
        L.orc_set_refstructure.restype = C.c_int
        L.orc_set_refstructure.argtypes = [C.c_void_p, C.c_int, C.c_int] + [C.POINTER(C.c_float)] * 4
        _lib = L
    return _lib


def philox(ctr, key):
    c = (C.c_uint32 * 4)(*ctr)
    k = (C.c_uint32 * 2)(*key)
    o = (C.c_uint32 * 4)()
    lib().orc_philox4x32_10(c, k, o)
    return list(o)


def spline_value(order: int, x: float) -> float:
    return lib().orc_spline_value(order, x)


def pppm_gfb(order: int) -> np.ndarray:
    """Coefficients of the PPPM alias-sum polynomial in sin^2(kh/2) (recpcal.F90:179-198)."""
    out = np.zeros(order)
    lib().orc_pppm_gfb(order, out.ctypes.data_as(C.POINTER(C.c_double)))
    return out


def binsearch(coord, v) -> int:
    c = A.as_f64(coord)
    return lib().orc_binsearch(A.ptr(c, C.c_double), len(c), float(v))


def enginit_mesh(hist: A.ErmodHist, numslv: int):
    L = lib()
    ermax, esmax = C.c_int32(), C.c_int32()
    rc = L.orc_enginit_mesh(C.byref(hist), numslv, None, None, None, None, C.byref(ermax), C.byref(esmax))
    if rc != 0:
        raise RuntimeError(f"mesh error {rc}")
    uvcrd = np.zeros(ermax.value)
    uvmax = np.zeros(numslv, dtype=np.int32)
    uvsoft = np.zeros(numslv, dtype=np.int32)
    escrd = np.zeros(esmax.value)
    L.orc_enginit_mesh(C.byref(hist), numslv, A.ptr(uvcrd, C.c_double), A.ptr(uvmax, C.c_int32),
                       A.ptr(uvsoft, C.c_int32), A.ptr(escrd, C.c_double), C.byref(ermax), C.byref(esmax))
    return uvcrd, uvmax, uvsoft, escrd


class Oracle:
    """Oracle context mirroring engclear / engconst / engstore."""

    def __init__(self, params: dict, topo, hist: dict | None = None, precision: int = 8, nthreads: int = 0):
        from ermod_openacc_b200 import systems as S
        self.L = lib()
        self.params = dict(params)
        self.topo = topo
        self.uvcrd, self.uvmax, self.uvsoft, self.escrd = enginit_mesh(S.hist_struct(hist), topo.numslv)
        self.ermax, self.esmax, self.numslv = len(self.uvcrd), len(self.escrd), topo.numslv
        self._ps = S.params_struct(self.params)
        self._ts, self._keep = topo.as_struct()
        self._ms = A.ErmodMesh(numslv=self.numslv, ermax=self.ermax, esmax=self.esmax,
                               uvcrd=A.ptr(self.uvcrd, C.c_double), uvmax=A.ptr(self.uvmax, C.c_int32),
                               uvsoft=A.ptr(self.uvsoft, C.c_int32), escrd=A.ptr(self.escrd, C.c_double))
        st = C.c_int()
        nth = nthreads or os.cpu_count() or 1
        self.h = self.L.orc_create(C.byref(self._ps), C.byref(self._ts), C.byref(self._ms), precision, nth,
                                   C.byref(st))
        if st.value != 0:
            msg = self.L.orc_last_error(self.h).decode()
            self.L.orc_destroy(self.h)
            self.h = None
            raise RuntimeError(f"oracle create failed {st.value} {msg}")
        phys = (topo.sluvid == A.PT_SOLVENT) | (topo.sluvid == A.PT_SOLUTE)
        self.slvmax = int(phys.sum())
        self.maxdst = params["maxins"] if params["slttype"] != A.SLT_SOLN else int((topo.sluvid > 0).sum())
        self.nsite_slt = int(topo.numsite[-1]) if params["slttype"] != A.SLT_SOLN else 0

    def __del__(self):
        if getattr(self, "h", None):
            self.L.orc_destroy(self.h)
            self.h = None

    def set_refstructure(self, refspec, host_crd, host_w, slt_crd, slt_w):
        hc, hw, sc, sw = (A.as_f32(x) for x in (host_crd, host_w, slt_crd, slt_w))
        self._ref = (hc, hw, sc, sw)
        rc = self.L.orc_set_refstructure(self.h, int(refspec), len(hw), A.ptr(hc, C.c_float), A.ptr(hw, C.c_float),
                                         A.ptr(sc, C.c_float), A.ptr(sw, C.c_float))
        if rc != 0:
            raise RuntimeError(f"oracle set_refstructure failed {rc} {self.L.orc_last_error(self.h).decode()}")
        return rc

    def engclear(self):
        self.L.orc_engclear(self.h)

    def engconst(self, stnum, sitepos, cell, wsys=1.0, ins_conf=None, ins_weight=None):
        sp = A.as_f32(sitepos)
        cl = A.as_f32(cell)
        ic = None if ins_conf is None else A.as_f32(ins_conf)
        iw = None if ins_weight is None else A.as_f32(ins_weight)
        fl = np.zeros(max(1, self.maxdst * self.numslv), dtype=np.float32)
        rc = self.L.orc_engconst(self.h, stnum, A.ptr(sp, C.c_float), A.ptr(cl, C.c_float), wsys,
                                 A.ptr(ic, C.c_float), A.ptr(iw, C.c_float), A.ptr(fl, C.c_float))
        self.flceng = fl
        return rc

    def last_error(self) -> str:
        return self.L.orc_last_error(self.h).decode()

    def uvengy(self):
        u = np.zeros(self.maxdst * self.slvmax)
        u0 = np.zeros(self.maxdst)
        self.L.orc_get_uvengy(self.h, A.ptr(u, C.c_double), A.ptr(u0, C.c_double))
        return u.reshape(self.maxdst, self.slvmax), u0

    def insertions(self):
        o = np.zeros(3 * self.nsite_slt * self.maxdst, dtype=np.float32)
        self.L.orc_get_insertions(self.h, A.ptr(o, C.c_float))
        return o

    def insertion_weights(self):
        w = np.zeros(self.maxdst)
        self.L.orc_get_insw(self.h, A.ptr(w, C.c_double))
        return w

    def engfac(self):
        K1, K2, K3 = self.params["ms1max"], self.params["ms2max"], self.params["ms3max"]
        o = np.zeros((K3, K2, K1 // 2 + 1))
        self.L.orc_get_engfac(self.h, A.ptr(o, C.c_double))
        return o

    def accum(self, normalise=False):
        ed = np.zeros(self.ermax)
        ec = np.zeros(self.ermax * self.ermax) if self.params["corrcal"] else None
        es = np.zeros(self.esmax) if self.params["selfcal"] else None
        sl = np.zeros(self.numslv, dtype=np.float32)
        mn = np.zeros(self.numslv + 1, dtype=np.float32)
        mx = np.zeros(self.numslv + 1, dtype=np.float32)
        acc = A.ErmodAccum(edens=A.ptr(ed, C.c_double), ecorr=A.ptr(ec, C.c_double),
                           eself=A.ptr(es, C.c_double), slnuv=A.ptr(sl, C.c_float),
                           minuv=A.ptr(mn, C.c_float), maxuv=A.ptr(mx, C.c_float))
        self.L.orc_fetch(self.h, C.byref(acc), 1 if normalise else 0)
        return dict(edens=ed, ecorr=None if ec is None else ec.reshape(self.ermax, self.ermax),
                    eself=es, slnuv=sl, minuv=mn, maxuv=mx, avslf=acc.avslf, engnorm=acc.engnorm,
                    engsmpl=acc.engsmpl, voffset=acc.voffset, voffset_initialized=acc.voffset_initialized)
