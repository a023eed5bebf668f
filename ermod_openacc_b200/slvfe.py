"""Solvation free energy from the energy distributions (slvfe's chmpot).

The downstream step of erdst: slvfe (slvfe/slvfe.F90) turns the solution
distribution rho (engsln), the reference-solvent distribution rho0 (engref)
and correlation chi0 (corref) into the solvation free energy with the
energy-representation functional.  This module evaluates that functional for
one data set with slvfe's defaults (slvfe/sfemain.F90:22-64):

  functional 'py-hnc', invmtrx 'reg', zerosft 'eczr', wgtfnform 'harm',
  extsln 'lin', extthres 1, minthres 0, normalize 'yes', slncor 'not',
  ljlrc 'not', uvread 'yes' (aveuv given), bins merged by `group` with inft 0.

Steps (slvfe.F90 line ranges):
  distnorm   1467-1542  rho, rho0 scaled to N per species; chi0 made
                        consistent with rho0 by the fixed-point row scaling
  getslncv   875-1001   omega_sln = -kT log(rho/rho0) - eps, linear
                        extrapolation into bins sampled on one side only
  getinscv   1003-1232  omega_ref from (chi0 - rho0 rho0^T + reg) x =
                        -kT (rho - rho0), Cholesky solve
  chmpot     744-803    the PY/HNC-interpolated functional per species

The arithmetic is FP64 on the host (the reference uses FP32).
"""
from __future__ import annotations

import numpy as np

__all__ = ["kT_of", "delta_mu", "delta_mu_gpu", "merge_bins", "representative_bins", "read_engfile", "read_corfile",
           "read_table", "delta_mu_from_files", "merge_mode", "merge_scan"]


def kT_of(temp_K: float) -> float:
    """kT in kcal/mol as slvfe computes it (slvfe.F90:272)."""
    return temp_K * 8.314510e-3 / 4.184


def _pyhnc_soln(f):
    with np.errstate(over="ignore", invalid="ignore", divide="ignore"):
        py = f + f / (np.exp(-f) - 1.0) + 1.0
    return np.where(f < 0.0, py, f / 2.0)


def _pyhnc_refs(f):
    with np.errstate(invalid="ignore", divide="ignore"):
        py = np.log1p(-f) * (1.0 / f - 1.0) + 1.0
    return np.where(f < 0.0, py, f / 2.0)


FUNCTIONALS = ("py-hnc", "hnc", "thnc", "none")


def _functional_terms(functional: str, omega, omega0, kT: float, et: float):
    """Per-bin integrands of the solution and reference-solvent sides (chmpot,
    slvfe.F90:759-774): py-hnc (pyhnc :1439-1465), hnc and thnc (thnc :1417-1436: half the
    indirect PMF over kT; thnc zeroes the reference side where its PMF lies below et),
    none (zero)."""
    f, f0 = omega / kT, omega0 / kT
    if functional == "py-hnc":
        return _pyhnc_soln(f), _pyhnc_refs(f0)
    if functional == "hnc":
        return f / 2.0, f0 / 2.0
    if functional == "thnc":
        return f / 2.0, np.where(omega0 < et, 0.0, f0 / 2.0)
    if functional == "none":
        return np.zeros_like(f), np.zeros_like(f0)
    raise ValueError(f"functional {functional!r}: one of {FUNCTIONALS}")


# posv_wrap's acceptance of the regularised Cholesky solve (slvfe.F90:478, 520-531): a larger
# residual or solution element sends getinscv to the eigen-decomposition (:1124-1170)
POSV_RESIDUAL = 1.0e-6
POSV_ABS = 1.0e6


def _normalise(edist, edens, ecorr, spec, nummol, tol=1.0e-8, itrmax=100):
    """distnorm: per-species scaling of rho and rho0, and the row scaling of chi0
    (a Gauss-Seidel sweep over the bins, as slvfe.F90:1503-1525 updates in place)."""
    rho = edist.copy()
    rho0 = edens.copy()
    nsp = len(nummol)
    masks = [spec == p for p in range(1, nsp + 1)]
    for p, m in enumerate(masks):
        s = rho[m].sum()
        rho[m] *= nummol[p] / s if s > 0.0 else 0.0
        s0 = rho0[m].sum()
        rho0[m] *= nummol[p] / s0 if s0 > 0.0 else 0.0
    chi = ecorr.copy()
    corr = np.ones(len(rho0))
    for it in range(itrmax + 1):
        for i in range(len(rho0)):
            acc = 0.0
            for p, m in enumerate(masks):
                a = float(np.dot(corr[m], chi[m, i]))
                if a > 0.0:
                    acc += nummol[p] / a
            corr[i] = acc / nsp * rho0[i]
        chi *= np.outer(corr, corr)
        err = np.max(np.abs(corr - 1.0)[rho0 > 0.0])
        if err <= tol:
            return rho, rho0, chi
        if it + 1 >= itrmax:
            break
    raise RuntimeError(f"chi0 normalisation did not converge (max correction {err:.3e})")


def _zero_bin(crd, dens, mask, tiny=1.0e-8):
    idx = np.nonzero(mask)[0]
    k = None
    for a, b in zip(idx[:-1], idx[1:]):
        if b != a + 1 or not (crd[a] <= 0.0 <= crd[b]):
            continue
        lo, hi = abs(crd[a]), crd[b]
        if hi > lo + tiny:
            k = a
        elif hi < lo - tiny:
            k = b
        else:
            k = a if dens[a] >= dens[b] else b
    if k is None:
        raise ValueError("the energy mesh has no bin pair around zero")
    return k


def core_counts(uvcrd, uvspec, tiny: float = 1.0e-8):
    """rduvcore per species as datread counts it from the bin coordinates (slvfe.F90:114-135):
    the bins since the spacing last stayed constant, i.e. the logarithmic core mesh."""
    crd = np.asarray(uvcrd, dtype=np.float64)
    spec = np.asarray(uvspec)
    out = {}
    for i in range(len(crd)):
        p = int(spec[i])
        if i == 0 or spec[i - 1] != p:
            cnt, core, prev_d = 1, 0, None
        else:
            cnt += 1
            d = crd[i] - crd[i - 1]
            if cnt > 2:
                core = 0 if abs(d - prev_d) < tiny else core + 1
            prev_d = d
        out[p] = core
    return out


def merge_groups(uvspec, group: int, core=None, inft: int = 0):
    """chmpot's bin grouping (slvfe.F90:609-640): per species, `group` consecutive bins form
    one merged bin; with inft the last rduvcore * inft / 100 bins of the core mesh go into
    the species' last merged bin too, which also takes the remainder.  Returns (merged index
    of every bin, start and end of every merged bin, 1 for the last merged bin of each species)."""
    spec = np.asarray(uvspec)
    n = len(spec)
    idr = np.zeros(n, dtype=np.int64)
    starts, ends, last = [], [], []
    i = 0
    while i < n:
        j = i
        while j < n and spec[j] == spec[i]:
            j += 1
        kc = (core[int(spec[i])] * inft) // 100 if inft else 0
        m = (j - i - kc) // group
        if m < 1:
            raise ValueError(f"species {spec[i]} has fewer bins than the group size {group}")
        idr[i:j] = len(starts) + np.minimum(np.arange(j - i) // group, m - 1)
        for q in range(m):
            starts.append(i + q * group)
            ends.append(i + (q + 1) * group if q < m - 1 else j)
            last.append(1 if q == m - 1 else 0)
        i = j
    return idr, np.array(starts), np.array(ends), np.array(last)


def merge_bins(edist, edens, ecorr, uvcrd, uvspec, group: int, inft: int = 0):
    """The merged distributions, correlation matrix, coordinates and species
    (slvfe.F90:642-698): sums over each group, the mean coordinate, and the species'
    last original coordinate for its last merged bin."""
    core = core_counts(uvcrd, uvspec) if inft else None
    idr, st, en, last = merge_groups(uvspec, group, core, inft)
    P = np.zeros((len(st), len(idr)))
    P[idr, np.arange(len(idr))] = 1.0
    crd = np.asarray(uvcrd, dtype=np.float64)
    mc = (P @ crd) / P.sum(axis=1)
    mc[last == 1] = crd[en[last == 1] - 1]
    chi = np.asarray(ecorr, dtype=np.float64)
    return (P @ np.asarray(edist, dtype=np.float64), P @ np.asarray(edens, dtype=np.float64), P @ chi @ P.T, mc,
            np.asarray(uvspec)[st])


def delta_mu(edist, edens, ecorr, uvcrd, uvspec, temp_K: float, aveuv, slfeng: float = 0.0, group: int = 1,
             inft: int = 0, functional: str = "py-hnc", et: float = 0.0):
    """(per-species solvation free energies, total) in kcal/mol.

    group > 1 first merges that many consecutive bins per species: chmpot's grouping with
    inft 0 (slvfe.F90:609-698).  The reference reports group pickgr = 3 in its range and
    merge modes (sfemain.F90:55, slvfe.F90:1647).  functional: 'py-hnc' (the default),
    'hnc', 'thnc' with threshold et (kcal/mol; sfemain.F90:177 selects thnc when et != 0)
    or 'none' (slvfe.F90:759-774)."""
    if functional not in FUNCTIONALS:
        raise ValueError(f"functional {functional!r}: one of {FUNCTIONALS}")
    # the sampled-bin thresholds use the smallest values of the data as read (slvfe.F90:884-885)
    rd_min = float(np.min(np.asarray(edist)[np.asarray(edist) > 0.0]))
    rr_min = float(np.min(np.asarray(edens)[np.asarray(edens) > 0.0]))
    if group > 1 or inft:
        edist, edens, ecorr, uvcrd, uvspec = merge_bins(edist, edens, ecorr, uvcrd, uvspec, group, inft)
    return _delta_mu(edist, edens, ecorr, uvcrd, uvspec, temp_K, aveuv, slfeng, rd_min, rr_min, functional, et)


def _delta_mu(edist, edens, ecorr, uvcrd, uvspec, temp_K: float, aveuv, slfeng: float, rd_min: float,
              rr_min: float, functional: str = "py-hnc", et: float = 0.0):
    """delta_mu on the mesh as given.

    edist: rho (solution, engstore-normalised); edens, ecorr: rho0 and chi0
    (reference solvent); uvcrd: bin coordinates; uvspec: 1-based species of
    each bin; aveuv: average solute-solvent energy per species in solution;
    slfeng: solute self energy (slfslt = 'yes')."""
    rd = np.asarray(edist, dtype=np.float64)
    rr = np.asarray(edens, dtype=np.float64)
    cr = np.asarray(ecorr, dtype=np.float64)
    crd = np.asarray(uvcrd, dtype=np.float64)
    spec = np.asarray(uvspec)
    nsp = int(spec.max())
    n = len(rd)
    kT = kT_of(temp_K)
    nummol = [float(np.rint(rd[spec == p].sum())) for p in range(1, nsp + 1)]
    rho, rho0, chi = _normalise(rd, rr, cr, spec, nummol)
    # omega in solution: direct where both distributions are sampled
    ratio_s = np.minimum(rho / rd_min, 10.0)
    ratio_r = np.minimum(rho0 / rr_min, 10.0)
    both = (np.rint(ratio_s) >= 1) & (np.rint(ratio_r) >= 1)
    omega = np.zeros(n)
    with np.errstate(divide="ignore", invalid="ignore"):
        omega[both] = -kT * np.log(rho[both] / rho0[both]) - crd[both]
    hsum = rho + rho0
    harm = np.where(hsum > 0.0, rho * rho0 / np.where(hsum > 0.0, hsum, 1.0), 0.0)
    for i in np.nonzero(~both)[0]:
        if rho[i] <= 0.0:
            omega[i] = 0.0
            continue
        same = (spec == spec[i]) & both
        lower = np.nonzero(same[:i])[0]
        upper = np.nonzero(same[i + 1:])[0] + i + 1
        m = lower[-1] if len(lower) else 0
        k = upper[0] if len(upper) else n - 1
        if both[m] and both[k]:
            j = m if abs(m - i) < abs(k - i) else k
        elif both[m] or both[k]:
            j = m if both[m] else k
        else:
            raise ValueError(f"cannot extrapolate omega at energy {crd[i]}")
        sel = np.nonzero(same)[0]
        shift = crd[sel] - crd[j]
        shift = np.where(sel < i, -shift - 2.0 * (crd[j] - crd[i]), shift)
        w = np.exp(-shift / kT) * harm[sel]
        keep = w > 0.0
        sel, w = sel[keep], w[keep] / w[keep].sum()
        x, y = crd[sel], omega[sel]
        m1, m2 = np.dot(w, x), np.dot(w, x * x)
        c0 = (m2 * np.dot(w, y) - m1 * np.dot(w, x * y)) / (m2 - m1 * m1)
        c1 = (np.dot(w, x * y) - m1 * np.dot(w, y)) / (m2 - m1 * m1)
        omega[i] = c0 + c1 * crd[i]
    # omega in the reference solvent: regularised correlation solve
    pos = rho0 > 0.0
    A = np.where(np.outer(pos, pos), chi - np.outer(rho0, rho0), 0.0)
    A[~pos, ~pos] = 1.0
    A[np.diag_indices(n)] = np.where(pos, np.diag(A), 1.0)
    ddiff = -kT * (rho - rho0)
    rhs = np.where(pos, ddiff, 0.0)
    Areg = A.copy()
    for p in range(1, nsp + 1):
        sp = pos & (spec == p)
        reg = np.trace(A[np.ix_(sp, sp)]) / sp.sum() ** 2
        Areg[np.ix_(sp, sp)] += reg
    x = None
    try:
        L = np.linalg.cholesky(Areg)
        x = np.linalg.solve(L.T, np.linalg.solve(L, rhs))
        if np.abs(Areg @ x - rhs).max() > POSV_RESIDUAL or np.abs(x).max() > POSV_ABS:
            x = None
    except np.linalg.LinAlgError:
        pass
    if x is None:
        val, vec = np.linalg.eigh(A)
        coef = (vec[pos, nsp:].T @ ddiff[pos]) / val[nsp:]
        x = vec[:, nsp:] @ coef
    zero_x = np.array([x[_zero_bin(crd, rho0, spec == p)] for p in range(1, nsp + 1)])
    with np.errstate(divide="ignore", invalid="ignore"):
        omega0 = np.where(pos, ddiff / np.where(pos, rho0, 1.0) - x, 0.0)
    omega0 += zero_x[spec - 1]
    # the functional
    live = (rho > 0.0) | (rho0 > 0.0)
    lcent = -(omega + crd)
    w = np.where(rho >= rho0, 1.0, 1.0 - ((rho - rho0) / np.where(hsum > 0.0, hsum, 1.0)) ** 2)
    lsln, lref = _functional_terms(functional, omega, omega0, kT, et)
    fac = w * lsln + (1.0 - w) * lref
    terms = -kT * (rho - rho0) + lcent * rho + kT * fac * (rho - rho0)
    chmpt = np.array([terms[live & (spec == p)].sum() for p in range(1, nsp + 1)]) + np.asarray(aveuv)
    return chmpt, float(chmpt.sum() + slfeng)


# ---------------------------------------------------------------------------
# erdst's output files (engproc.F90:630-722) as slvfe reads them
# ---------------------------------------------------------------------------
def representative_bins(uvcrd, uvmax, uvsoft):
    """representative_bin_info (engproc.F90:1355-1387) for every bin: (left, middle,
    1/width, 1-based species); the last bin of a species has width 0 (1/width = 0)."""
    c = np.asarray(uvcrd, dtype=np.float64)
    left = c.copy()
    middle = c.copy()
    invwt = np.zeros(len(c))
    spec = np.zeros(len(c), dtype=int)
    base = 0
    for p, (mx, sf) in enumerate(zip(uvmax, uvsoft)):
        for idpt in range(1, mx + 1):
            i = base + idpt - 1
            spec[i] = p + 1
            if i + 1 >= len(c):
                continue
            if idpt <= sf:
                middle[i] = (c[i] + c[i + 1]) / 2.0
                invwt[i] = 1.0 / (c[i + 1] - c[i])
            elif idpt < mx:
                middle[i] = np.sqrt(c[i] * c[i + 1])
                invwt[i] = 1.0 / (c[i + 1] - c[i])
        base += mx
    return left, middle, invwt, spec


def _fortran_real(tok: str) -> float:
    """A real as Fortran list-directed input takes it, including the exponent form
    without a letter ("0.1234567-100") that E editing writes beyond two exponent digits."""
    t = tok.strip()
    try:
        return float(t)
    except ValueError:
        k = max(t.rfind("+"), t.rfind("-"))
        if k > 0 and t[k - 1] not in "eEdD":
            return float(t[:k] + "E" + t[k:])
        return float(t.replace("D", "E").replace("d", "e"))


def read_engfile(path) -> dict:
    """engsln / engref (engproc.F90:686-699): one header line, then bin_left,
    bin_middle, species, ratio (= the engstore-normalised distribution) and dens
    (ratio / bin width) per bin, as slvfe's datread takes them (slvfe.F90:380-386)."""
    rows = []
    with open(path) as f:
        f.readline()
        for line in f:
            if line.strip():
                rows.append([_fortran_real(t) for t in line.split()])
    a = np.array(rows)
    return dict(left=a[:, 0], middle=a[:, 1], spec=a[:, 2].astype(int), ratio=a[:, 3], dens=a[:, 4])


def read_corfile(path, ermax: int) -> np.ndarray:
    """corsln / corref: one Fortran unformatted record of ermax x ermax FP64 values
    (engproc.F90:702-713, read by slvfe.F90:404-407), column-major."""
    raw = open(path, "rb").read()
    n = ermax * ermax * 8
    head = int(np.frombuffer(raw[:4], dtype="<i4")[0])
    tail = int(np.frombuffer(raw[4 + n:8 + n], dtype="<i4")[0]) if len(raw) >= n + 8 else -1
    if head != n or tail != n or len(raw) != n + 8:
        raise ValueError(f"{path}: not one record of {ermax}x{ermax} FP64 values")
    return np.frombuffer(raw[4:4 + n], dtype="<f8").reshape(ermax, ermax, order="F").copy()


def read_table(path) -> np.ndarray:
    """Numeric rows of aveuv.tt, weight_soln / weight_refs and the like (list-directed)."""
    rows = []
    with open(path) as f:
        for line in f:
            t = line.split()
            if t and not t[0].startswith("#"):
                try:
                    rows.append([_fortran_real(x) for x in t])
                except ValueError:
                    continue   # a text header line (uvrange.tt)
    return np.array(rows)


def delta_mu_gpu(edist, edens, ecorr, uvcrd, uvspec, temp_K: float, aveuv, slfeng: float = 0.0,
                 device: int = 0, group: int = 1, inft: int = 0, functional: str = "py-hnc", et: float = 0.0,
                 evd: bool = True, info: dict | None = None):
    """delta_mu on the GPU (include/ermod_slvfe.h, ermod_slvfe_delta_mu_ex): the same
    functional, options and arguments, FP64 CUDA kernels, with getinscv's eigen-decomposition
    fallback (evd=False reports slv_chl instead).  Raises RuntimeError with slvfe's failure
    name; `info`, if given, receives {"used_evd": bool}."""
    import ctypes as C
    from . import _capi as A
    if functional not in A.SLVFE_FUNCTIONALS:
        raise ValueError(f"functional {functional!r}: one of {tuple(A.SLVFE_FUNCTIONALS)}")
    lib = A.load_library()
    rd = A.as_f64(edist)
    rr = A.as_f64(edens)
    chi = np.asfortranarray(np.asarray(ecorr, dtype=np.float64))
    crd = A.as_f64(uvcrd)
    spec = np.ascontiguousarray(uvspec, dtype=np.int32)
    av = A.as_f64(np.atleast_1d(aveuv))
    nsp = int(spec.max())
    out = np.zeros(nsp)
    tot = C.c_double()
    used = C.c_int32()
    opts = A.ErmodSlvfeOpts(functional=A.SLVFE_FUNCTIONALS[functional], evd=1 if evd else 0, et=float(et))
    rc = lib.ermod_slvfe_delta_mu_ex(device, len(rd), nsp, group, inft, A.ptr(rd, C.c_double), A.ptr(rr, C.c_double),
                                     chi.ctypes.data_as(C.POINTER(C.c_double)), A.ptr(crd, C.c_double),
                                     A.ptr(spec, C.c_int32), kT_of(temp_K), A.ptr(av, C.c_double), float(slfeng),
                                     C.byref(opts), A.ptr(out, C.c_double), C.byref(tot), C.byref(used))
    if info is not None:
        info["used_evd"] = bool(used.value)
    if rc != 0:
        raise RuntimeError(f"{lib.ermod_slvfe_last_error().decode()} ({rc})")
    return out, tot.value


def delta_mu_from_files(soln_dir, refs_dir, temp_K: float, suffix: str = "tt", slfslt: bool = False,
                        group: int = 1):
    """slvfe on one division's files: engsln.<suffix> and aveuv.tt from the solution run,
    engref.<suffix> and corref.<suffix> from the reference-solvent run; with slfslt the
    solute self energy is weight_refs' third column averaged with its first-column
    weights (slvfe.F90:257-286).  Returns delta_mu's (per-species, total)."""
    import os
    sln = read_engfile(os.path.join(soln_dir, f"engsln.{suffix}"))
    ref = read_engfile(os.path.join(refs_dir, f"engref.{suffix}"))
    if not np.array_equal(sln["spec"], ref["spec"]) or not np.allclose(sln["middle"], ref["middle"]):
        raise ValueError("solution and reference-solvent meshes differ")
    chi = read_corfile(os.path.join(refs_dir, f"corref.{suffix}"), len(ref["ratio"]))
    av = read_table(os.path.join(soln_dir, "aveuv.tt"))
    div = 1 if suffix == "tt" else int(suffix)
    aveuv = av[div - 1, 1:]
    slf = 0.0
    if slfslt:
        wr = read_table(os.path.join(refs_dir, "weight_refs"))
        w = wr[:, 1] / wr[:, 1].sum()
        slf = float(np.dot(w, wr[:, 2]))
    return delta_mu(sln["ratio"], ref["ratio"], chi, sln["middle"], sln["spec"], temp_K, aveuv, slf, group=group)


def _suffixes(directory, prefix):
    import os
    names = [f for f in os.listdir(directory) if f.startswith(prefix + ".")]
    nums = sorted(int(f.split(".")[1]) for f in names if f.split(".")[1].isdigit())
    if nums:
        return [f"{n:02d}" for n in nums]
    if prefix + ".tt" in names:
        return ["tt"]
    raise FileNotFoundError(f"no {prefix} files in {directory}")


# (group, inft) of slvfe's default parameter sets (slvfe.F90:177-199)
PARAMS_INFCHK_NOT = tuple((g, 0) for g in range(1, 6))
PARAMS_INFCHK_YES = ((1, 0), (1, 60), (1, 80), (1, 100), (2, 0), (3, 0), (4, 0), (5, 0), (5, 60), (5, 80), (5, 100))


def merge_scan(soln_dir, refs_dir, temp_K: float, numdiv: int = 0, infchk: bool = False, pickgr: int = 3,
               slfslt: bool = False, gpu: bool = False, device: int = 0) -> dict:
    """slvfe's merge mode over its default parameter sets (numprm 5 with infchk 'not', 11 with
    'yes'; slvfe.F90:177-199): the table per (group, inft), and the headline at
    (pickgr, inft 0) (sfemain.F90:55, slvfe.F90:1647)."""
    sets = PARAMS_INFCHK_YES if infchk else PARAMS_INFCHK_NOT
    table = {(g, i): merge_mode(soln_dir, refs_dir, temp_K, numdiv, g, slfslt, gpu, device, inft=i) for g, i in sets}
    if (pickgr, 0) not in table:
        raise ValueError(f"pickgr {pickgr} is not among the parameter sets")
    return dict(table=table, picked=table[(pickgr, 0)], pickgr=pickgr)


def merge_mode(soln_dir, refs_dir, temp_K: float, numdiv: int = 0, group: int = 3, slfslt: bool = False,
               gpu: bool = False, device: int = 0, inft: int = 0) -> dict:
    """slvfe's clcond 'merge' for one (group, inft 0): the solution runs engsln.NN split into
    numdiv blocks, each block's distribution and aveuv the weight_soln-weighted mean of its
    runs; the reference-solvent runs engref.NN / corref.NN merged over all runs with
    weight_refs (refmerge 'yes'); delta mu per block, their mean and the 95 % error
    2 s / sqrt(n) with the n / (n - 1) variance (datread slvfe.F90:292-444, wrtmerge
    :1733-1790).  numdiv <= 0 or >= the number of runs takes every run as a block; a count
    that does not divide it moves up to the next divisor (sfemain.F90:148-153)."""
    import os
    ssuf = _suffixes(soln_dir, "engsln")
    rsuf = _suffixes(refs_dir, "engref")
    numsln, numref = len(ssuf), len(rsuf)
    if numdiv <= 0 or numdiv >= numsln:
        numdiv = numsln
    while numsln % numdiv:
        numdiv += 1
    def weights(path, n):
        if os.path.exists(path):
            t = read_table(path)
            return t[:n, 1].astype(np.float64), t
        return np.ones(n), None
    wsln, _ = weights(os.path.join(soln_dir, "weight_soln"), numsln)
    wref, wref_tab = weights(os.path.join(refs_dir, "weight_refs"), numref)
    wref = wref / wref.sum()
    refs = [read_engfile(os.path.join(refs_dir, f"engref.{s}")) for s in rsuf]
    middle, spec = refs[0]["middle"], refs[0]["spec"]
    n = len(middle)
    rr = sum(w * r["ratio"] for w, r in zip(wref, refs))
    chi = sum(w * read_corfile(os.path.join(refs_dir, f"corref.{s}"), n) for w, s in zip(wref, rsuf))
    slf = 0.0
    if slfslt:
        if wref_tab is None or wref_tab.shape[1] < 3:
            raise ValueError("slfslt needs the self energies of weight_refs")
        slf = float(np.dot(wref, wref_tab[:numref, 2]))
    uvene = read_table(os.path.join(soln_dir, "aveuv.tt"))[:numsln, 1:]
    per = numsln // numdiv
    f = delta_mu_gpu if gpu else delta_mu
    kw = dict(device=device) if gpu else {}
    blocks = []
    for b in range(numdiv):
        idx = range(b * per, (b + 1) * per)
        w = wsln[list(idx)] / wsln[list(idx)].sum()
        runs = [read_engfile(os.path.join(soln_dir, f"engsln.{ssuf[i]}")) for i in idx]
        if any(not np.array_equal(r["spec"], spec) or not np.allclose(r["left"], refs[0]["left"]) for r in runs):
            raise ValueError("solution and reference-solvent energy coordinates are inconsistent")
        rd = sum(wi * r["ratio"] for wi, r in zip(w, runs))
        aveuv = w @ uvene[list(idx)]
        blocks.append(f(rd, rr, chi, middle, spec, temp_K, aveuv, slf, group=group, inft=inft, **kw)[1])
    blocks = np.array(blocks)
    mean = float(blocks.mean())
    err = None
    if numdiv > 1:
        std = np.sqrt(numdiv / (numdiv - 1.0)) * np.sqrt(max((blocks ** 2).mean() - mean ** 2, 0.0))
        err = float(2.0 * std / np.sqrt(numdiv))
    return dict(blocks=blocks, mean=mean, error95=err, numdiv=numdiv, group=group, inft=inft)
