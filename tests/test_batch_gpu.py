"""CUDA-graph frames and solute batches: bit-identical to direct, separate runs.

A frame replayed as a captured graph runs the same kernels with the same
arguments as direct launches, and a batch member runs its own unchanged
pipeline on its own graph branch, so every result must match bit for bit.
"""
import numpy as np
import pytest

from ermod_openacc_b200 import Batch, Engine
from ermod_openacc_b200 import systems as S

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lib(engine_lib):
    return engine_lib


def run_frames(eng, w, frames):
    for fr in frames:
        pos, cell = w.frame(fr)
        assert eng.engconst(fr + 1, pos, cell) >= 0
    return eng.uvengy(), eng.accum()


def assert_same(ra, rb):
    (ua, u0a), aa = ra
    (ub, u0b), ab = rb
    np.testing.assert_array_equal(ua, ub)
    np.testing.assert_array_equal(u0a, u0b)
    for k in ("edens", "ecorr", "minuv", "maxuv"):
        if aa[k] is not None:
            np.testing.assert_array_equal(aa[k], ab[k])
    for k in ("engnorm", "avslf", "engsmpl", "voffset"):
        assert aa[k] == ab[k]


@pytest.mark.parametrize("path", [1, 2, 3])
def test_graph_frames_match_direct_launches(lib, path):
    w = S.make_workload(2, small=True, maxins=96)
    res = []
    for mode in ({"graph_mode": 0}, {"graph_mode": 1}, {"stage_timing": 1}):
        eng = Engine(dict(w.params, keep_uvengy=1, spectrum_path=path, **mode), w.topo, w.hist)
        res.append(run_frames(eng, w, range(4)))
        eng.close()
    assert_same(res[0], res[1])
    assert_same(res[0], res[2])


def test_batch_members_match_separate_runs(lib):
    ws = S.make_batch_workloads(4, small=True, maxins=[64, 32, 96, 40], site_range=(10, 70))
    frames = range(3)
    alone = []
    for w in ws:
        eng = Engine(dict(w.params, keep_uvengy=1), w.topo, w.hist)
        alone.append(run_frames(eng, w, frames))
        eng.close()
    members = [Engine(dict(w.params, keep_uvengy=1), w.topo, w.hist) for w in ws]
    batch = Batch(members)
    for fr in frames:
        pos, cell = ws[0].frame(fr)
        assert batch.engconst(fr + 1, pos, cell) >= 0
    assert batch.last_ms() > 0
    for m, ref in zip(members, alone):
        assert_same((m.uvengy(), m.accum()), ref)
    batch.close()
    for m in members:
        m.close()


def test_batch_rejects_mismatched_solvent(lib):
    a = S.make_workload(2, small=True, maxins=32)
    b = S.make_workload(1, small=True)
    ea = Engine(a.params, a.topo, a.hist)
    eb = Engine(b.params, b.topo, b.hist)
    with pytest.raises(Exception):
        Batch([ea, eb])
    with pytest.raises(Exception):
        Batch([ea, ea])


def test_contexts_of_different_sizes_coexist(engine_lib):
    """Kernel shared-memory limits are per-device attributes shared by every context: a context
    created later for a smaller solute must not lower them below what an earlier context with a
    larger solute launches with (real-space solute tiles, direct-sum site tiles)."""
    big = S.make_batch_workloads(1, small=True, maxins=32, site_range=(64, 64))[0]
    eb = Engine(big.params, big.topo, big.hist)
    small = S.make_workload(2, small=True, maxins=32)
    es = Engine(small.params, small.topo, small.hist)
    assert eb.nsite_slt == 64 and es.nsite_slt == 12
    assert eb.engconst(1, *big.frame(0)) >= 0
    assert es.engconst(1, *small.frame(0)) >= 0
    assert eb.engconst(2, *big.frame(1)) >= 0
    eb.close()
    es.close()
