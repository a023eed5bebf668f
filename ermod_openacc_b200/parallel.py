"""engstore's cross-rank step: the reference's MPI reduction at the end of a
division (erdst/engproc.F90:538-602), over torch.distributed.

Frames (or insertions) are independent, so ranks run their own engines with
no exchange inside a frame; a division ends with

  1. voffset: max over ranks, and each rank's histograms rescaled by
     exp(-/+(voffset_local - voffset_max)/kT) (refs / soln) when wgtslf is on
     (engproc.F90:541-575); avslf is not rescaled, as in the reference;
  2. sums of avslf, engnorm, engsmpl, eself, slnuv, edens, ecorr
     (engproc.F90:580-595), min / max of minuv / maxuv (engproc.F90:597-602).

The reference reduces to rank 0; here every rank receives the result, which
rank 0 then normalises exactly as engstore does.  The sums are formed in rank
order from an all-gather of every rank's partials, so every rank holds the same
bits and the result does not depend on the collective's internal reduction order
(ring or tree, which a library may pick by size and rank count); minima and maxima,
which are exact in any order, use an all-reduce.  The communicator is any
torch.distributed group: NCCL for device tensors, gloo for host tensors.
"""
from __future__ import annotations

import math

import numpy as np

from . import _capi as A


def reduce_accumulators(acc: dict, slttype: int, wgtslf: int, temp: float, group=None, device=None) -> dict:
    """Raw accumulators of this rank (Engine.accum()) -> the division's totals over all ranks."""
    import torch
    import torch.distributed as dist
    dev = torch.device(device) if device is not None else torch.device("cpu")
    out = {k: (None if v is None else (np.array(v, copy=True) if isinstance(v, np.ndarray) else v))
           for k, v in acc.items()}
    if wgtslf:
        v_local = float(acc["voffset"])
        t = torch.tensor([v_local], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
        v_max = float(t.item())
        if not acc.get("voffset_initialized", 1):
            v_local = v_max            # an empty rank must not produce NaN
        sign = 1.0 if slttype == A.SLT_SOLN else -1.0
        scale = math.exp(sign * (v_local - v_max) / temp)
        out["engnorm"] = acc["engnorm"] * scale
        for k in ("edens", "ecorr", "eself"):
            if out[k] is not None:
                out[k] = out[k] * scale
        if slttype == A.SLT_SOLN and out["slnuv"] is not None:
            out["slnuv"] = out["slnuv"] * scale
        out["voffset"] = v_max

    nrank = dist.get_world_size(group=group)

    def allsum(x, op=None):
        if x is None:
            return None
        arr = np.asarray(x, dtype=np.float64)
        t = torch.from_numpy(np.ascontiguousarray(arr)).to(dev)
        if op is not None:                      # MIN / MAX: exact in any order
            dist.all_reduce(t, op=op, group=group)
            r = t.cpu().numpy()
        else:                                   # SUM: in rank order, the same on every rank
            parts = [torch.empty_like(t) for _ in range(nrank)]
            dist.all_gather(parts, t, group=group)
            r = parts[0].cpu().numpy().copy()
            for p in parts[1:]:
                r += p.cpu().numpy()
        return r if arr.ndim else float(r)

    for k in ("avslf", "engnorm", "engsmpl"):
        out[k] = allsum(out[k])
    for k in ("eself", "slnuv", "edens", "ecorr"):
        if out[k] is not None:
            out[k] = allsum(out[k]).reshape(np.shape(acc[k]))
    if out.get("minuv") is not None:
        out["minuv"] = allsum(out["minuv"], dist.ReduceOp.MIN).astype(np.float32)
        out["maxuv"] = allsum(out["maxuv"], dist.ReduceOp.MAX).astype(np.float32)
    return out


def normalise(tot: dict, slttype: int, temp: float):
    """engstore's normalisation (engproc.F90:609-628) of reduced totals: (normalised dict, avediv[2])."""
    out = dict(tot)
    nrm = tot["engnorm"]
    out["edens"] = tot["edens"] / nrm
    if tot.get("ecorr") is not None:
        out["ecorr"] = tot["ecorr"] / nrm
    if tot.get("eself") is not None:
        out["eself"] = tot["eself"] / nrm
    avslf = tot["avslf"] / nrm
    out["avslf"] = avslf
    if slttype == A.SLT_SOLN:
        if tot.get("slnuv") is not None:
            out["slnuv"] = np.asarray(tot["slnuv"], dtype=np.float64) / nrm   # aveuv (engproc.F90:622)
        av2 = tot["voffset"] - temp * math.log(avslf)
    else:
        av2 = tot["voffset"] + temp * math.log(avslf)
    return out, np.array([nrm / tot["engsmpl"], av2])


def engstore_all(engine, group=None, device=None):
    """engstore over every rank of `group`: reduce this rank's engine accumulators and normalise."""
    p = engine.params
    tot = reduce_accumulators(engine.accum(), p["slttype"], p["wgtslf"], p["temp"], group, device)
    return normalise(tot, p["slttype"], p["temp"])
