"""engstore's cross-rank reduction on two gloo ranks (CPU).

Each rank accumulates its own insertions with its own voffset (its first
insertion's self energy); after the reduction the normalised distributions
and avediv must equal those of one process that saw every insertion, because
the voffset rescale makes the weights of all ranks commensurate."""
import math
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from ermod_openacc_b200 import _capi as A
from ermod_openacc_b200 import parallel as PR

TEMP = 300.0 * 8.314510e-3 / 4.184
NBIN = 40


def make_insertions(seed=0, n=60):
    rng = np.random.default_rng(seed)
    u0 = rng.normal(0.0, 1.5, n)
    cnt = rng.poisson(3.0, size=(n, NBIN)).astype(np.float64)
    return u0, cnt


def accumulate(u0, cnt, slttype):
    """update_histogram's sums (engproc.F90:883-962) with voffset = the first u0."""
    v = u0[0]
    sign = 1.0 if slttype == A.SLT_SOLN else -1.0
    w = np.exp(sign * (u0 - v) / TEMP)
    return dict(edens=w @ cnt, ecorr=(cnt * w[:, None]).T @ cnt, eself=None, slnuv=None,
                minuv=np.array([-1.0, float(cnt.min())], np.float32), maxuv=np.array([2.0, float(cnt.max())], np.float32),
                avslf=float(len(u0)), engnorm=float(w.sum()), engsmpl=float(len(u0)), voffset=float(v),
                voffset_initialized=1)


def _rank(rank, port, slttype, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=2)
    u0, cnt = make_insertions()
    half = len(u0) // 2
    sl = slice(0, half) if rank == 0 else slice(half, None)
    acc = accumulate(u0[sl], cnt[sl], slttype)
    tot = PR.reduce_accumulators(acc, slttype, 1, TEMP)
    norm, avediv = PR.normalise(tot, slttype, TEMP)
    if rank == 0:
        np.savez(out, edens=norm["edens"], ecorr=norm["ecorr"], avediv=avediv, engsmpl=tot["engsmpl"],
                 minuv=norm["minuv"], maxuv=norm["maxuv"])
    dist.barrier()
    dist.destroy_process_group()


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("slttype", [A.SLT_REFS_RIGID, A.SLT_SOLN])
def test_two_rank_reduction_matches_one_process(tmp_path, slttype):
    out = str(tmp_path / "r.npz")
    mp.spawn(_rank, args=(free_port(), slttype, out), nprocs=2, join=True)
    r = np.load(out)
    u0, cnt = make_insertions()
    one, avediv = PR.normalise(accumulate(u0, cnt, slttype), slttype, TEMP)
    np.testing.assert_allclose(r["edens"], one["edens"], rtol=1e-12)
    np.testing.assert_allclose(r["ecorr"], one["ecorr"], rtol=1e-12)
    np.testing.assert_allclose(r["avediv"], avediv, rtol=1e-12, atol=1e-12)
    assert r["engsmpl"] == len(u0)
    assert r["minuv"][1] == cnt.min() and r["maxuv"][1] == cnt.max()


def _rank_sum(rank, port, nrank, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=nrank)
    rng = np.random.default_rng(100 + rank)
    acc = dict(edens=rng.normal(size=NBIN) * 10.0 ** rng.uniform(-8, 8, NBIN), ecorr=None, eself=None, slnuv=None,
               minuv=None, maxuv=None, avslf=float(rng.normal()), engnorm=float(rng.normal() * 1e6),
               engsmpl=float(rank + 1), voffset=0.0, voffset_initialized=1)
    tot = PR.reduce_accumulators(acc, A.SLT_REFS_RIGID, 0, TEMP)
    np.savez(out + f".{rank}.npz", edens=tot["edens"], engnorm=tot["engnorm"])
    dist.barrier()
    dist.destroy_process_group()


def test_sums_are_in_rank_order_and_identical_on_every_rank(tmp_path):
    """Three gloo ranks with partials spread over 16 decades: every rank gets the same bits, and
    they are the sequential sum in rank order."""
    out = str(tmp_path / "s")
    mp.spawn(_rank_sum, args=(free_port(), 3, out), nprocs=3, join=True)
    res = [np.load(out + f".{r}.npz") for r in range(3)]
    expect = None
    for r in range(3):
        rng = np.random.default_rng(100 + r)
        e = rng.normal(size=NBIN) * 10.0 ** rng.uniform(-8, 8, NBIN)
        expect = e.copy() if expect is None else expect + e
    for r in range(3):
        np.testing.assert_array_equal(res[r]["edens"], expect)
        assert res[r]["engnorm"] == res[0]["engnorm"]

