"""ermod_histogram_noalloc against the engine's own histogram (GPU).

The entry point exists for hosts that may not allocate GPU memory: it must
give the same edens as ermod_engconst's binning for the same energies, and
keep doing so on the next call, since every call reuses the same fixed
device array (what must start at zero is cleared each call).  This file is
collected last so a failure here leaves the rest of the suite already run.
"""
import ctypes as C

import numpy as np
import pytest

from ermod_openacc_b200 import Engine
from ermod_openacc_b200 import _capi as A
from ermod_openacc_b200 import systems as S

pytestmark = pytest.mark.gpu


def call_noalloc(lib, eng, u, weight, device=0, spec=None, mesh=None, slttype=None):
    if spec is None:
        spec = eng.topo.uvspec[(eng.topo.sluvid == A.PT_SOLVENT) | (eng.topo.sluvid == A.PT_SOLUTE)]
    spec = np.ascontiguousarray(spec, dtype=np.int32)
    uvcrd, uvmax, uvsoft = mesh if mesh is not None else (eng.uvcrd, eng.uvmax, eng.uvsoft)
    uvcrd = np.ascontiguousarray(uvcrd, dtype=np.float64)
    uvmax = np.ascontiguousarray(uvmax, dtype=np.int32)
    uvsoft = np.ascontiguousarray(uvsoft, dtype=np.int32)
    out = np.full(len(uvcrd), np.nan)
    uu = np.ascontiguousarray(u, dtype=np.float64)
    ww = np.ascontiguousarray(weight, dtype=np.float64)
    st = eng.params["slttype"] if slttype is None else slttype
    rc = lib.ermod_histogram_noalloc(device, st, A.ptr(uu, C.c_double), uu.shape[0],
                                     uu.shape[1], A.ptr(spec, C.c_int32), A.ptr(uvcrd, C.c_double),
                                     A.ptr(uvmax, C.c_int32), A.ptr(uvsoft, C.c_int32), len(uvmax),
                                     A.ptr(ww, C.c_double), A.ptr(out, C.c_double))
    return rc, out


def test_noalloc_matches_engine_twice(engine_lib):
    lib = engine_lib
    w = S.make_workload(2, small=True, maxins=96)
    # unit weights (no self-energy weighting, constant volume): edens is the plain count
    prm = dict(w.params, keep_uvengy=1, wgtslf=0, estype=A.ES_NVT)
    eng = Engine(prm, w.topo, w.hist)
    for call in range(2):
        eng.engclear()
        pos, cell = w.frame(call)
        assert eng.engconst(call + 1, pos, cell) >= 0
        u, _ = eng.uvengy()
        ref = eng.accum()["edens"]
        rc, got = call_noalloc(lib, eng, u, np.ones(u.shape[0]))
        assert rc >= 0
        np.testing.assert_allclose(got, ref, rtol=1e-12, atol=0.0)
        assert got.sum() == pytest.approx(u.shape[0] * u.shape[1], rel=1e-12)


def test_noalloc_soln_matches_engine_twice(engine_lib):
    """Solute in solution: the engine skips the solute's own molecule, so the caller leaves
    that column out; the per-species energy sums the binning kernel forms in this mode live
    in the fixed array too."""
    lib = engine_lib
    w = S.make_workload(1, small=True)
    prm = dict(w.params, keep_uvengy=1, wgtslf=0, estype=A.ES_NVT)
    eng = Engine(prm, w.topo, w.hist)
    spec = eng.topo.uvspec[(eng.topo.sluvid == A.PT_SOLVENT) | (eng.topo.sluvid == A.PT_SOLUTE)]
    keep = spec > 0
    assert keep.sum() == len(spec) - 1
    for call in range(2):
        eng.engclear()
        pos, cell = w.frame(call)
        assert eng.engconst(call + 1, pos, cell) >= 0
        u, _ = eng.uvengy()
        ref = eng.accum()["edens"]
        rc, got = call_noalloc(lib, eng, u[:, keep], np.ones(u.shape[0]), spec=spec[keep])
        assert rc >= 0
        np.testing.assert_allclose(got, ref, rtol=1e-12, atol=0.0)
        assert got.sum() == pytest.approx(u.shape[0] * keep.sum(), rel=1e-12)


def test_noalloc_small_mesh_leaves_engine_launchable(engine_lib):
    """A call on a coarse mesh must not lower the binning kernel's shared-memory limit below
    what an engine with a finer mesh, created earlier, launches with."""
    lib = engine_lib
    w = S.make_workload(2, small=True, maxins=32)
    prm = dict(w.params, keep_uvengy=1, wgtslf=0, estype=A.ES_NVT)
    eng = Engine(prm, w.topo, w.hist)
    pos, cell = w.frame(0)
    assert eng.engconst(1, pos, cell) >= 0
    u, _ = eng.uvengy()
    coarse = np.concatenate([[-1.0e9], np.linspace(-40.0, 40.0, 62), [1.0e30]])
    rc, got = call_noalloc(lib, eng, u, np.ones(u.shape[0]),
                           mesh=(coarse, [len(coarse)], [len(coarse)]))
    assert rc >= 0 and got.sum() == pytest.approx(u.size, rel=1e-12)
    eng.engclear()
    assert eng.engconst(2, *w.frame(1)) >= 0
    assert eng.accum()["edens"].sum() == pytest.approx(u.size, rel=1e-12)


def test_noalloc_rejects_oversized_request(engine_lib):
    lib = engine_lib
    w = S.make_workload(2, small=True, maxins=8)
    eng = Engine(w.params, w.topo, w.hist)
    nmol = eng.slvmax
    ntarget = A.NOALLOC_SCRATCH_BYTES // (8 * nmol) + 1   # the energies alone exceed the array
    u = np.zeros((ntarget, nmol))
    rc, _ = call_noalloc(lib, eng, u, np.ones(ntarget))
    assert rc == A.ERMOD_ERR_OVERFLOW
