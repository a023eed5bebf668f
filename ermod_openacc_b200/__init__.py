"""B200-native (sm_100a) energy-distribution engine for ERmod's erdst.

The engine replaces erdst's per-frame hot path (realcal, insertion,
recpcal, engproc binning and ecorr) with CUDA kernels behind the C-ABI in
include/ermod_b200.h.  `Engine` mirrors engclear / engconst / engstore.
"""
from ._capi import load_library  # noqa: F401
from .engine import Batch, Engine, ErmodError, enginit_mesh  # noqa: F401
from . import systems  # noqa: F401
