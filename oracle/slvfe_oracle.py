"""TEST INFRASTRUCTURE, NOT PRODUCT CODE: a CPU restatement of slvfe's
solvation free energy for the checker (tests/ only).

Follows slvfe/slvfe.F90 with the defaults of slvfe/sfemain.F90:22-64 for a
single data set (clcond 'basic', inft 0; group 1 makes the bin mapping of
chmpot the identity, larger groups go through merge_bins): functional 'py-hnc', invmtrx 'reg', zerosft
'eczr', wgtfnform 'harm', wgtf2smpl 'yes', extsln 'lin', extthres 1,
minthres 0, normalize 'yes', slncor 'not', ljlrc 'not', uvread 'yes'.
Written with explicit loops in the reference's order, in FP64.

The reference cannot run here (nvfortran only), so this restatement is
pinned by the identities the tests check, not by reference outputs.
"""
from __future__ import annotations

import numpy as np


def kT_of(temp_K: float) -> float:
    """kT in kcal/mol (slvfe.F90:272)."""
    return temp_K * 8.314510e-3 / 4.184


def _pyhnc(indpmf: float, cnt: int, kT: float) -> float:
    """slvfe.F90:1439-1465."""
    factor = indpmf / kT
    if cnt in (1, 2):
        if factor < 0.0:
            if cnt == 1:
                intg = factor + factor / (np.exp(-factor) - 1.0)
            else:
                intg = np.log(1.0 - factor) * (1.0 / factor - 1.0)
            intg += 1.0
        else:
            intg = factor / 2.0
    else:
        if factor > 0.0:
            intg = 1.0 - np.log(1.0 + factor) * (1.0 / factor + 1.0)
        else:
            intg = -factor / 2.0
    return intg


def _thnc(indpmf: float, et: float, cnt: int, kT: float) -> float:
    """slvfe.F90:1417-1436."""
    factor = indpmf / kT
    if cnt == 2 and indpmf < et:
        factor = 0.0
    return factor / 2.0


def _sfewgt(fsln: float, fref: float) -> float:
    """slvfe.F90:1402-1414."""
    if fsln >= fref:
        return 1.0
    factor = (fsln - fref) / (fsln + fref)
    return 1.0 - factor ** 2


def _distnorm(edist, edens, ecorr, uvspec, nummol, numslv, norm_error=1.0e-8, itrmax=100):
    """slvfe.F90:1467-1542 with slncor = 'not'."""
    gemax = len(edist)
    out = []
    for cnt in (1, 2):
        edhst = (edist if cnt == 1 else edens).copy()
        for pti in range(1, numslv + 1):
            mask = uvspec == pti
            factor = edhst[mask].sum()
            factor = nummol[pti - 1] / factor if factor > 0.0 else 0.0
            edhst[mask] *= factor
        if cnt == 1:
            out.append(edhst)
            continue
        edmcr = ecorr.copy()             # edmcr[iduvp, iduv] as the Fortran (column-major) matrix
        errtmp = norm_error + 1.0
        itrcnt = 0
        correc = np.ones(gemax)
        while errtmp > norm_error and itrcnt <= itrmax:
            for iduv in range(gemax):
                lcsln = 0.0
                for pti in range(1, numslv + 1):
                    mask = uvspec == pti
                    ampl = np.sum(correc[mask] * edmcr[mask, iduv])
                    if ampl > 0.0:
                        lcsln += nummol[pti - 1] / ampl
                lcsln /= numslv
                correc[iduv] = lcsln * edhst[iduv]
            edmcr *= np.outer(correc, correc)
            errtmp = np.max(np.abs(correc - 1.0)[edhst > 0.0])
            itrcnt += 1
            if itrcnt >= itrmax:
                raise RuntimeError(f"correlation-matrix normalisation did not converge ({errtmp})")
        out.append(edhst)
        out.append(edmcr)
    return out[0], out[1], out[2]


def _zeroec(pti, edvec, uvcrd, uvspec, tiny=1.0e-8):
    """slvfe.F90:1319-1357 (cnt selects which distribution breaks ties)."""
    k = None
    for iduv in range(len(uvcrd) - 1):
        if uvspec[iduv] == pti and uvcrd[iduv] <= 0.0 <= uvcrd[iduv + 1]:
            factor = abs(uvcrd[iduv])
            ampl = uvcrd[iduv + 1]
            if ampl > factor + tiny:
                k = iduv
            elif ampl < factor - tiny:
                k = iduv + 1
            else:
                k = iduv if edvec[iduv] >= edvec[iduv + 1] else iduv + 1
    if k is None:
        raise RuntimeError("no zero-energy bin")
    return k


def _rduvcore(rdcrd, rdspec, tiny=1.0e-8):
    """datread's count of the core (non-uniformly spaced) bins per species (slvfe.F90:114-135)."""
    rduvmax, rduvcore = {}, {}
    k = 0
    crdprev = crddif_prev = 0.0
    for iduv in range(len(rdcrd)):
        pti, crdnow = int(rdspec[iduv]), float(rdcrd[iduv])
        if pti != k:
            rduvmax[pti] = 1
            rduvcore[pti] = 0
            k = pti
        else:
            rduvmax[pti] += 1
            crddif_now = crdnow - crdprev
            if rduvmax[pti] > 2:
                if abs(crddif_now - crddif_prev) < tiny:
                    rduvcore[pti] = 0
                else:
                    rduvcore[pti] += 1
            crddif_prev = crddif_now
        crdprev = crdnow
    return rduvcore


def merge_bins(rddst, rddns, rdcor, rdcrd, rdspec, group, inft=0):
    """chmpot's grouping of `group` consecutive bins per species (slvfe.F90:609-698), the
    last rduvcore * inft / 100 core bins joining the last merged bin, in the reference's
    loop order, 1-based indices as there."""
    rddst, rddns, rdcor = (np.asarray(x, dtype=np.float64) for x in (rddst, rddns, rdcor))
    rdcrd = np.asarray(rdcrd, dtype=np.float64)
    rdspec = np.asarray(rdspec)
    ermax = len(rddst)
    numslv = int(rdspec.max())
    rduvmax = [0] * (numslv + 1)
    for iduv in range(ermax):
        rduvmax[int(rdspec[iduv])] += 1
    rduvcore = _rduvcore(rdcrd, rdspec)
    uvmax = [0] * (numslv + 1)
    idrduv = [0] * (ermax + 1)
    gemax = 0
    for pti in range(1, numslv + 1):
        k = rduvcore[pti] * inft // 100
        m = (rduvmax[pti] - k) // group
        uvmax[pti] = m
        gemax += m
        if pti == 1:
            cnt, j = 1, 0
        else:
            cnt, j = 1 + sum(rduvmax[1:pti]), sum(uvmax[1:pti])
        for iduv in range(cnt, cnt + rduvmax[pti]):
            k = (iduv - cnt) // group + 1
            if k >= m:
                k = m
            idrduv[iduv] = k + j
    uvcrd = [0.0] * (gemax + 1)
    gpnum = [0] * (gemax + 1)
    uvspec = [0] * (gemax + 1)
    for iduv in range(1, ermax + 1):
        k = idrduv[iduv]
        uvcrd[k] += rdcrd[iduv - 1]
        gpnum[k] += 1
        uvspec[k] = int(rdspec[iduv - 1])
    for k in range(1, gemax + 1):
        if gpnum[k] > 0:
            uvcrd[k] /= gpnum[k]
    cnt, k = rduvmax[1], uvmax[1]
    for pti in range(1, numslv + 1):
        if pti > 1:
            cnt += rduvmax[pti]
            k += uvmax[pti]
        uvcrd[k] = rdcrd[cnt - 1]
    edist = [0.0] * (gemax + 1)
    edens = [0.0] * (gemax + 1)
    for iduv in range(1, ermax + 1):
        k = idrduv[iduv]
        edist[k] += rddst[iduv - 1]
        edens[k] += rddns[iduv - 1]
    ecorr = np.zeros((gemax + 1, gemax + 1))
    for iduv in range(1, ermax + 1):
        k = idrduv[iduv]
        for iduvp in range(1, ermax + 1):
            ecorr[idrduv[iduvp], k] += rdcor[iduvp - 1, iduv - 1]
    return (np.array(edist[1:]), np.array(edens[1:]), ecorr[1:, 1:], np.array(uvcrd[1:]),
            np.array(uvspec[1:]))


def delta_mu(edist, edens, ecorr, uvcrd, uvspec, temp_K, aveuv, slfeng=0.0, group=1, inft=0, functional="py-hnc",
             et=0.0):
    """Solvation free energy (kcal/mol) per solvent species and in total.

    edist  solution energy distribution per bin (engsln), edens / ecorr the
    reference-solvent distribution and correlation (engref / corref), all as
    engstore writes them; uvcrd the bin coordinates, uvspec the species of
    each bin (1-based); aveuv the average solute-solvent energy per species
    in solution, slfeng the solute self energy added with slfslt = 'yes'.
    group merges that many consecutive bins per species first (chmpot, slvfe.F90:609-698).
    Returns (chmpt[numslv], total)."""
    # getslncv's thresholds use the smallest sampled values of the data as read (slvfe.F90:884-885)
    min_rddst = np.asarray(edist, dtype=np.float64)[np.asarray(edist) > 0.0].min()
    min_rddns = np.asarray(edens, dtype=np.float64)[np.asarray(edens) > 0.0].min()
    if group > 1 or inft:
        edist, edens, ecorr, uvcrd, uvspec = merge_bins(edist, edens, ecorr, uvcrd, uvspec, group, inft)
    rddst = np.asarray(edist, dtype=np.float64)
    rddns = np.asarray(edens, dtype=np.float64)
    rdcor = np.asarray(ecorr, dtype=np.float64)
    uvcrd = np.asarray(uvcrd, dtype=np.float64)
    uvspec = np.asarray(uvspec)
    numslv = int(uvspec.max())
    gemax = len(rddst)
    kT = kT_of(temp_K)
    # number of molecules per species from the solution distribution (datread, slvfe.F90:425-444)
    nummol = [float(np.rint(rddst[uvspec == pti].sum())) for pti in range(1, numslv + 1)]
    edist_, edens_, ecorr_ = _distnorm(rddst, rddns, rdcor, uvspec, nummol, numslv)
    # ---- getslncv (slvfe.F90:875-1001), extsln = 'lin', zerosft = 'eczr' ----
    ext = np.ones(gemax, dtype=bool)
    for iduv in range(gemax):
        j = min(10, int(np.rint(edist_[iduv] / min_rddst))) if edist_[iduv] / min_rddst <= 10 else 10
        k = min(10, int(np.rint(edens_[iduv] / min_rddns))) if edens_[iduv] / min_rddns <= 10 else 10
        if j < 1 or k < 1:
            ext[iduv] = False
    slncv = np.zeros(gemax)
    for iduv in range(gemax):
        if ext[iduv]:
            slncv[iduv] = -kT * np.log(edist_[iduv] / edens_[iduv]) - uvcrd[iduv]
    for iduv in range(gemax):
        if ext[iduv]:
            continue
        if edist_[iduv] <= 0.0:
            slncv[iduv] = 0.0
            continue
        pti = uvspec[iduv]
        m, k = 0, gemax - 1
        for p in range(iduv):
            if uvspec[p] == pti and ext[p] and m < p:
                m = p
        for p in range(gemax - 1, iduv, -1):
            if uvspec[p] == pti and ext[p] and k > p:
                k = p
        if ext[m] and ext[k]:
            j = m if abs(m - iduv) < abs(k - iduv) else k
        elif ext[m]:
            j = m
        elif ext[k]:
            j = k
        else:
            raise RuntimeError(f"extrapolation not possible at {uvcrd[iduv]}")
        work = np.zeros(gemax)
        for p in range(gemax):
            if uvspec[p] == pti and ext[p]:
                factor = uvcrd[p] - uvcrd[j]
                if p < iduv:
                    factor = -factor - 2.0 * (uvcrd[j] - uvcrd[iduv])
                fs, fr = edist_[p], edens_[p]
                wght = fs * fr / (fs + fr) if fs + fr > 0.0 else 0.0      # wgtdst 'harm'
                work[p] = np.exp(-factor / kT) * wght
        pos = work > 0.0
        work /= work[pos].sum()
        mat11 = np.sum(work[pos] * uvcrd[pos])
        mat22 = np.sum(work[pos] * uvcrd[pos] ** 2)
        mat12 = np.sum(work[pos] * slncv[pos])
        mat21 = np.sum(work[pos] * uvcrd[pos] * slncv[pos])
        a0 = (mat22 * mat12 - mat11 * mat21) / (mat22 - mat11 ** 2)
        a1 = (mat21 - mat11 * mat12) / (mat22 - mat11 ** 2)
        slncv[iduv] = a0 + a1 * uvcrd[iduv]
    zrsln = np.zeros(numslv)             # 'eczr': no shift
    # ---- getinscv (slvfe.F90:1003-1232), invmtrx = 'reg', zerosft = 'eczr' ----
    edvec = edens_
    edmcr = ecorr_.copy()
    for iduv in range(gemax):
        for p in range(gemax):
            if edvec[p] > 0.0 and edvec[iduv] > 0.0:
                edmcr[p, iduv] = edmcr[p, iduv] - edvec[p] * edvec[iduv]
            else:
                edmcr[p, iduv] = 1.0 if p == iduv else 0.0
    ddiff = -kT * (edist_ - edens_)
    inv = edmcr.copy()
    work = ddiff.copy()
    work[edvec <= 0.0] = 0.0
    regfac = np.zeros(numslv)
    regcnt = np.zeros(numslv)
    for iduv in range(gemax):
        if edvec[iduv] > 0.0:
            regfac[uvspec[iduv] - 1] += edmcr[iduv, iduv]
            regcnt[uvspec[iduv] - 1] += 1.0
    regfac = regfac / regcnt / regcnt
    for iduv in range(gemax):
        if edvec[iduv] > 0.0:
            pti = uvspec[iduv]
            for p in range(gemax):
                if uvspec[p] == pti and edvec[p] > 0.0:
                    inv[p, iduv] += regfac[pti - 1]
    inscv = None
    try:
        L = np.linalg.cholesky(inv)
        inscv = np.linalg.solve(L.T, np.linalg.solve(L, work))
        # posv_wrap (slvfe.F90:520-531): residual above 1e-6 or an element above 1e6 is a failure
        residual = np.abs(inv @ inscv - work)
        if residual.max() > 1.0e-6 or np.abs(inscv).max() > 1.0e6:
            inscv = None
    except np.linalg.LinAlgError:
        pass
    if inscv is None:                 # EVD fallback (slvfe.F90:1124-1170)
        egnval, vec = np.linalg.eigh(edmcr)
        inscv = np.zeros(gemax)
        for i in range(numslv, gemax):
            inscv += vec[:, i] * (np.sum((ddiff * vec[:, i])[edvec > 0.0]) / egnval[i])
    zerouv = np.array([inscv[_zeroec(pti, edvec, uvcrd, uvspec)] for pti in range(1, numslv + 1)])
    for iduv in range(gemax):
        inscv[iduv] = ddiff[iduv] / edvec[iduv] - inscv[iduv] if edvec[iduv] > 0.0 else 0.0
    for pti in range(1, numslv + 1):
        inscv[uvspec == pti] -= -zerouv[pti - 1]
    # ---- chmpot (slvfe.F90:744-803) ----
    chmpt = np.zeros(numslv)
    for pti in range(1, numslv + 1):
        slvfe = 0.0
        for iduv in range(gemax):
            if uvspec[iduv] != pti:
                continue
            if edist_[iduv] <= 0.0 and edens_[iduv] <= 0.0:
                continue
            slvfe -= kT * (edist_[iduv] - edens_[iduv])
            lcent = -(slncv[iduv] + zrsln[pti - 1] + uvcrd[iduv])
            slvfe += lcent * edist_[iduv]
            if functional == "py-hnc":
                lcsln = _pyhnc(slncv[iduv], 1, kT)
                lcref = _pyhnc(inscv[iduv], 2, kT)
            elif functional == "hnc":
                lcsln = _thnc(slncv[iduv], -np.inf, 1, kT)
                lcref = _thnc(inscv[iduv], -np.inf, 2, kT)
            elif functional == "thnc":
                lcsln = _thnc(slncv[iduv], et, 1, kT)
                lcref = _thnc(inscv[iduv], et, 2, kT)
            elif functional == "none":
                lcsln = lcref = 0.0
            else:
                raise ValueError(functional)
            ampl = _sfewgt(edist_[iduv], edens_[iduv])
            factor = ampl * lcsln + (1.0 - ampl) * lcref
            slvfe += kT * factor * (edist_[iduv] - edens_[iduv])
        chmpt[pti - 1] = slvfe + aveuv[pti - 1]
    return chmpt, float(chmpt.sum() + slfeng)
