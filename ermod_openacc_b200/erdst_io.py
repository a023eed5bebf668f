"""erdst's on-disk formats through the library's C-ABI (include/ermod_io.h).

Trajectory reading stands in for trajectory.F90 over vmdfio.c (the VMD
molfile plugin path) for DCD files; `write_engstore` writes engstore's files
(engproc.F90:630-722).  Readers of those files for the slvfe step are in
`ermod_openacc_b200.slvfe`.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import _capi as A

__all__ = ["Trajectory", "IOError_", "write_engstore", "fortran_format", "rmsd_bestfit"]


class IOError_(RuntimeError):
    def __init__(self, code: int, name: str):
        super().__init__(f"{name} ({code})")
        self.code = code
        self.name = name


def _lib():
    return A.load_library()


def _check(rc: int) -> int:
    if rc < 0:
        raise IOError_(rc, _lib().ermod_io_last_error().decode())
    return rc


class Trajectory:
    """open_trajectory / read_trajectory / close_trajectory (trajectory.F90:39-91)."""

    def __init__(self, path: str | os.PathLike):
        self.lib = _lib()
        h = C.c_void_p()
        na, nf, hc = C.c_int32(), C.c_int32(), C.c_int32()
        _check(self.lib.ermod_traj_open(os.fsencode(path), C.byref(h), C.byref(na), C.byref(nf), C.byref(hc)))
        self.h = h
        self.path = os.fspath(path)
        self.natoms, self.nframes, self.has_cell = na.value, nf.value, bool(hc.value)
        self._crd = np.zeros(3 * self.natoms, dtype=np.float32)
        self._cell = np.zeros(9, dtype=np.float32)

    def read(self, natoms: int | None = None):
        """Next frame as (crd [3*natoms] float32, cell [9] float32 column-major), or None past the end."""
        n = self.natoms if natoms is None else natoms
        if n != self.natoms:
            self._crd = np.zeros(3 * n, dtype=np.float32)
        rc = _check(self.lib.ermod_traj_read(self.h, n, A.ptr(self._crd, C.c_float), A.ptr(self._cell, C.c_float)))
        if rc == A.TRJ_EOF:
            return None
        return self._crd.copy(), self._cell.copy()

    def rewind(self):
        _check(self.lib.ermod_traj_rewind(self.h))

    def close(self):
        if getattr(self, "h", None):
            self.lib.ermod_traj_close(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        self.close()


def write_engstore(directory, params: dict, mesh: dict, norm: dict, division: int, engdiv: int,
                   avediv, aveuv=None):
    """engstore's files for one division (engproc.F90:630-722).

    params: slttype, corrcal, selfcal, wgtslf; mesh: uvcrd, uvmax, uvsoft, escrd;
    norm: the normalised accumulators (edens, ecorr, eself, minuv, maxuv) as
    returned by Engine.engstore; avediv [engdiv, 2] and aveuv [engdiv, numslv]
    (soln) of every division so far.
    """
    lib = _lib()
    uvcrd = A.as_f64(mesh["uvcrd"])
    uvmax = np.ascontiguousarray(mesh["uvmax"], dtype=np.int32)
    uvsoft = np.ascontiguousarray(mesh["uvsoft"], dtype=np.int32)
    escrd = A.as_f64(mesh["escrd"]) if mesh.get("escrd") is not None else None
    keep = []

    def f64(x):
        if x is None:
            return None
        a = A.as_f64(x)
        keep.append(a)
        return A.ptr(a, C.c_double)

    def f32(x):
        if x is None:
            return None
        a = A.as_f32(x)
        keep.append(a)
        return A.ptr(a, C.c_float)

    info = A.ErmodStoreInfo(slttype=params["slttype"], corrcal=params["corrcal"], selfcal=params["selfcal"],
                            wgtslf=params["wgtslf"], division=division, engdiv=engdiv, numslv=len(uvmax),
                            ermax=len(uvcrd), esmax=0 if escrd is None else len(escrd),
                            uvcrd=A.ptr(uvcrd, C.c_double), uvmax=A.ptr(uvmax, C.c_int32),
                            uvsoft=A.ptr(uvsoft, C.c_int32), escrd=A.ptr(escrd, C.c_double))
    ec = norm.get("ecorr") if params["corrcal"] else None
    if ec is not None:   # the dict holds the column-major buffer viewed row-major: flatten it back as is
        ec = np.ascontiguousarray(ec, dtype=np.float64).reshape(-1)
    acc = A.ErmodAccum(edens=f64(norm["edens"]), ecorr=f64(ec),
                       eself=f64(norm.get("eself") if params["selfcal"] else None),
                       minuv=f32(norm.get("minuv")), maxuv=f32(norm.get("maxuv")))
    av = None if avediv is None else np.asarray(avediv, dtype=np.float64).reshape(engdiv, 2).ravel(order="F")
    au = None if aveuv is None else np.asarray(aveuv, dtype=np.float32).reshape(engdiv, -1).ravel(order="F")
    _check(lib.ermod_write_engstore(os.fsencode(os.fspath(directory)), C.byref(info), C.byref(acc), f64(av),
                                    f32(au)))


def fortran_format(kind: str, x: float, w: int, d: int = 0) -> str:
    """One value through a Fortran output edit descriptor: kind 'G', 'E', 'F' or 'I'."""
    buf = C.create_string_buffer(w + 1)
    _check(_lib().ermod_io_format("GEFI".index(kind), float(x), w, d, buf, w + 1))
    return buf.value.decode()


def rmsd_bestfit(ref, crd, w) -> float:
    """rmsd_bestfit (bestfit.F90:339-346) through the library."""
    r, c, ww = A.as_f32(ref).ravel(), A.as_f32(crd).ravel(), A.as_f32(w).ravel()
    v = _lib().ermod_rmsd_bestfit(len(ww), A.ptr(r, C.c_float), A.ptr(c, C.c_float), A.ptr(ww, C.c_float))
    if v < 0:
        raise IOError_(-1, "bst_zrw")
    return v
