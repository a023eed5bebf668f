"""ctypes mirror of include/ermod_b200.h.

The structs here must match the C header field for field; the library's
own loader (`load_library`) refuses to run without the CUDA build, so no
call made through this module can silently fall back to a CPU path.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

ERMOD_OK = 0
ERMOD_WARN_MBIN = 1
ERMOD_ERR_ARG = -1
ERMOD_ERR_CUDA = -2
ERMOD_ERR_ENG_MIN = -10
ERMOD_ERR_ENG_SFT = -11
ERMOD_ERR_ENG_CNS = -12
ERMOD_ERR_RCP_CNS = -13
ERMOD_ERR_INS_GEO = -14
ERMOD_ERR_ENG_ECD = -15
ERMOD_ERR_CELL = -16
ERMOD_ERR_OVERFLOW = -17
ERMOD_ERR_UNSUPPORTED = -20

SLT_SOLN, SLT_REFS_RIGID, SLT_REFS_FLEX = 1, 2, 3
PT_SOLVENT, PT_SOLUTE, PT_TEST_RIGID, PT_TEST_FLEX = 0, 1, 2, 3
SYS_NONPERIODIC, SYS_PERIODIC = 0, 1
ES_NVT, ES_NPT = 1, 2
EL_COULOMB, EL_EWALD, EL_PME, EL_PPPM = 0, 1, 2, 3
LJSWT_POT_CHM, LJSWT_POT_GMX, LJSWT_FRC_CHM, LJSWT_FRC_GMX = 0, 1, 2, 3
INSPOS_RANDOM, INSPOS_NOCHANGE = 0, 1
INSPOS_SPHERE, INSPOS_SLAB_GENERIC, INSPOS_SLAB_SYMMETRIC = 2, 3, 4
INSPOS_RMSD, INSPOS_GAUSS = 5, 6
INSSTR_NOREJECT, INSSTR_RMSD = 0, 1
INSROT_RANDOM, INSROT_NOCHANGE = 0, 1
PROPOSAL_UNIFORM, PROPOSAL_LEARNED = 0, 1

_i32p = C.POINTER(C.c_int32)
_f32p = C.POINTER(C.c_float)
_f64p = C.POINTER(C.c_double)


class ErmodParams(C.Structure):
    _fields_ = [
        ("slttype", C.c_int32), ("boxshp", C.c_int32), ("estype", C.c_int32),
        ("cltype", C.c_int32), ("ljswitch", C.c_int32),
        ("splodr", C.c_int32), ("ms1max", C.c_int32), ("ms2max", C.c_int32), ("ms3max", C.c_int32),
        ("maxins", C.c_int32),
        ("corrcal", C.c_int32), ("selfcal", C.c_int32), ("wgtslf", C.c_int32),
        ("insposition", C.c_int32), ("insorient", C.c_int32),
        ("iseed", C.c_int32),
        ("temp", C.c_double),
        ("elecut", C.c_float), ("lwljcut", C.c_float), ("upljcut", C.c_float), ("screen", C.c_float),
        ("ins_chunk", C.c_int32), ("ecorr_batch", C.c_int32), ("weight_bits", C.c_int32),
        ("proposal", C.c_int32),
        ("keep_uvengy", C.c_int32), ("ecorr_path", C.c_int32), ("spectrum_path", C.c_int32),
        ("graph_mode", C.c_int32), ("stage_timing", C.c_int32),
        ("lwreg", C.c_float), ("upreg", C.c_float), ("hostspec", C.c_int32),
        ("insstructure", C.c_int32), ("lwstr", C.c_float), ("upstr", C.c_float),
    ]


class ErmodTopology(C.Structure):
    _fields_ = [
        ("nummol", C.c_int32),
        ("numsite", _i32p), ("sluvid", _i32p), ("uvspec", _i32p),
        ("charge", _f32p), ("ljtype", _i32p), ("sitemass", _f32p),
        ("ljtype_max", C.c_int32),
        ("ljene_mat", _f32p), ("ljlensq_mat", _f32p),
        ("bfcoord", _f32p),
    ]


class ErmodMesh(C.Structure):
    _fields_ = [
        ("numslv", C.c_int32), ("ermax", C.c_int32), ("esmax", C.c_int32),
        ("uvcrd", _f64p), ("uvmax", _i32p), ("uvsoft", _i32p), ("escrd", _f64p),
    ]


class ErmodHist(C.Structure):
    _fields_ = [
        ("ecdmin", C.c_double), ("ecfmns", C.c_double), ("ecdcen", C.c_double),
        ("eccore", C.c_double), ("ecdmax", C.c_double),
        ("eclbin", C.c_double), ("ecfbin", C.c_double), ("ec0bin", C.c_double),
        ("finfac", C.c_double),
        ("pecore", C.c_int32),
    ]


class ErmodAccum(C.Structure):
    _fields_ = [
        ("edens", _f64p), ("ecorr", _f64p), ("eself", _f64p),
        ("slnuv", _f32p), ("minuv", _f32p), ("maxuv", _f32p),
        ("avslf", C.c_double), ("engnorm", C.c_double), ("engsmpl", C.c_double),
        ("voffset", C.c_double), ("voffset_initialized", C.c_int32),
    ]


class ErmodStoreInfo(C.Structure):
    _fields_ = [
        ("slttype", C.c_int32), ("corrcal", C.c_int32), ("selfcal", C.c_int32), ("wgtslf", C.c_int32),
        ("division", C.c_int32), ("engdiv", C.c_int32),
        ("numslv", C.c_int32), ("ermax", C.c_int32), ("esmax", C.c_int32),
        ("uvcrd", _f64p), ("uvmax", _i32p), ("uvsoft", _i32p), ("escrd", _f64p),
    ]


ERR_IO, ERR_FORMAT, TRJ_EOF = -30, -31, 1


def ptr(a, ctype):
    """Pointer to the data of a contiguous numpy array (None -> NULL)."""
    if a is None:
        return None
    return a.ctypes.data_as(C.POINTER(ctype))


PKG_DIR = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG_DIR, "libermod_b200.so")

# Every symbol include/*.h declares, with its ctypes signature.
class ErmodSlvfeOpts(C.Structure):
    """ermod_slvfe_opts (include/ermod_slvfe.h)."""
    _fields_ = [("functional", C.c_int32), ("evd", C.c_int32), ("et", C.c_double)]


SLVFE_FUNCTIONALS = {"py-hnc": 0, "hnc": 1, "thnc": 2, "none": 3}

SIGNATURES = {
    "ermod_abi_version": (C.c_int32, []),
    "ermod_enginit_mesh": (C.c_int32, [C.POINTER(ErmodHist), C.c_int32, _f64p, _i32p, _i32p, _f64p, _i32p, _i32p]),
    "ermod_create": (C.c_int32, [C.POINTER(C.c_void_p), C.c_int32, C.POINTER(ErmodParams),
                                 C.POINTER(ErmodTopology), C.POINTER(ErmodMesh)]),
    "ermod_engclear": (C.c_int32, [C.c_void_p]),
    "ermod_set_refstructure": (C.c_int32, [C.c_void_p, C.c_int32, C.c_int32, _f32p, _f32p, _f32p, _f32p]),
    "ermod_engconst": (C.c_int32, [C.c_void_p, C.c_int32, _f32p, _f32p, C.c_float, _f32p, _f32p, _f32p]),
    "ermod_engconst_dev": (C.c_int32, [C.c_void_p, C.c_int32, C.c_void_p, _f32p, C.c_float,
                                       C.c_void_p, C.c_void_p]),
    "ermod_fetch_accum": (C.c_int32, [C.c_void_p, C.POINTER(ErmodAccum)]),
    "ermod_engstore": (C.c_int32, [C.c_void_p, C.POINTER(ErmodAccum), _f64p]),
    "ermod_get_uvengy": (C.c_int32, [C.c_void_p, _f64p, _f64p]),
    "ermod_get_insertions": (C.c_int32, [C.c_void_p, _f32p, _f64p]),
    "ermod_get_sizes": (C.c_int32, [C.c_void_p, _i32p, _i32p, _i32p, _i32p]),
    "ermod_last_error": (C.c_char_p, [C.c_void_p]),
    "ermod_get_timings": (C.c_int32, [C.c_void_p, _f32p, C.c_int32]),
    "ermod_get_launch_count": (C.c_int64, [C.c_void_p]),
    "ermod_get_paths": (C.c_int32, [C.c_void_p, C.POINTER(C.c_int32), C.POINTER(C.c_int32)]),
    "ermod_batch_create": (C.c_int32, [C.POINTER(C.c_void_p), C.c_int32, C.POINTER(C.c_void_p)]),
    "ermod_batch_engconst": (C.c_int32, [C.c_void_p, C.c_int32, C.POINTER(C.c_float), C.POINTER(C.c_float),
                                         C.c_float]),
    "ermod_batch_engconst_dev": (C.c_int32, [C.c_void_p, C.c_int32, C.c_void_p, C.POINTER(C.c_float), C.c_float]),
    "ermod_batch_last_ms": (C.c_float, [C.c_void_p]),
    "ermod_batch_last_error": (C.c_char_p, [C.c_void_p]),
    "ermod_batch_destroy": (None, [C.c_void_p]),
    "ermod_proposal_config": (C.c_int32, [C.c_void_p, C.c_int32, C.c_int32, C.c_float, C.POINTER(C.c_float)]),
    "ermod_get_insertion_samples": (C.c_int32, [C.c_void_p, C.POINTER(C.c_float), C.POINTER(C.c_double),
                                                C.POINTER(C.c_int32)]),
    "ermod_mlp_create": (C.c_int32, [C.POINTER(C.c_void_p), C.c_int32, C.c_int32, C.POINTER(C.c_float)]),
    "ermod_mlp_nparams": (C.c_int32, []),
    "ermod_mlp_forward": (C.c_int32, [C.c_void_p, C.POINTER(C.c_float), C.c_int32, C.POINTER(C.c_float)]),
    "ermod_mlp_activations": (C.c_int32, [C.c_void_p, C.c_int32, C.POINTER(C.c_float)]),
    "ermod_mlp_gradients": (C.c_int32, [C.c_void_p, C.POINTER(C.c_float), C.POINTER(C.c_float), C.c_int32,
                                        C.POINTER(C.c_float), C.POINTER(C.c_double)]),
    "ermod_mlp_train_step": (C.c_int32, [C.c_void_p, C.POINTER(C.c_float), C.POINTER(C.c_float), C.c_int32,
                                         C.c_float, C.POINTER(C.c_double)]),
    "ermod_mlp_get_params": (C.c_int32, [C.c_void_p, C.POINTER(C.c_float)]),
    "ermod_mlp_destroy": (None, [C.c_void_p]),
    "ermod_destroy": (None, [C.c_void_p]),
    "ermod_histogram_noalloc": (C.c_int32, [C.c_int32, C.c_int32, _f64p, C.c_int32, C.c_int32, _i32p, _f64p,
                                            _i32p, _i32p, C.c_int32, _f64p, _f64p]),
    # include/ermod_io.h
    "ermod_traj_open": (C.c_int32, [C.c_char_p, C.POINTER(C.c_void_p), _i32p, _i32p, _i32p]),
    "ermod_traj_read": (C.c_int32, [C.c_void_p, C.c_int32, _f32p, _f32p]),
    "ermod_traj_rewind": (C.c_int32, [C.c_void_p]),
    "ermod_traj_close": (None, [C.c_void_p]),
    "ermod_write_engstore": (C.c_int32, [C.c_char_p, C.POINTER(ErmodStoreInfo), C.POINTER(ErmodAccum), _f64p,
                                         _f32p]),
    "ermod_io_format": (C.c_int32, [C.c_int32, C.c_double, C.c_int32, C.c_int32, C.c_char_p, C.c_int32]),
    "ermod_io_last_error": (C.c_char_p, []),
    "ermod_rmsd_bestfit": (C.c_double, [C.c_int32, _f32p, _f32p, _f32p]),
    # include/ermod_slvfe.h
    "ermod_slvfe_delta_mu": (C.c_int32, [C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32, _f64p, _f64p,
                                         _f64p, _f64p,
                                         _i32p,
                                         C.c_double, _f64p, C.c_double, _f64p, _f64p]),
    "ermod_slvfe_delta_mu_ex": (C.c_int32, [C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32, _f64p, _f64p,
                                            _f64p, _f64p, _i32p, C.c_double, _f64p, C.c_double,
                                            C.POINTER(ErmodSlvfeOpts), _f64p, _f64p, _i32p]),
    "ermod_slvfe_last_error": (C.c_char_p, []),
}

NOALLOC_SCRATCH_BYTES = 32 << 20

_LIB = None


def load_library(path: str | None = None):
    """Load libermod_b200.so (the CUDA build).  Raises if it is missing."""
    global _LIB
    if _LIB is not None and path is None:
        return _LIB
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise RuntimeError(f"libermod_b200.so not built ({p}); run __graft_entry__.build()")
    lib = C.CDLL(p)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if lib.ermod_abi_version() != 3:
        raise RuntimeError("libermod_b200.so ABI mismatch")
    if path is None:
        _LIB = lib
    return lib


def as_f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def as_f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def as_i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)
