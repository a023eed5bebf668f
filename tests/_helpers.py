"""Shared helpers of the parity tests (test-side only)."""
from __future__ import annotations

import numpy as np

from ermod_openacc_b200 import _capi as A
from ermod_openacc_b200 import systems as S

# Per-molecule energy tolerance against the FP64 oracle: 1e-5 relative plus
# 2e-5 kcal/mol absolute (a tenth of the finest bin width, 2e-4 kcal/mol).
RTOL = 1e-5
ATOL = 2e-5


def energy_tol(e_ref):
    return RTOL * np.abs(e_ref) + ATOL


def phys_uvspec(topo: S.Topology):
    phys = (topo.sluvid == A.PT_SOLVENT) | (topo.sluvid == A.PT_SOLUTE)
    return topo.uvspec[phys]


def bins_of(E, uvcrd, uvmax, spec):
    """getiduv (engproc.F90:1111-1171): 0-based global bin = idmin + count(edges < E) - 1."""
    off = np.concatenate([[0], np.cumsum(uvmax)])
    out = np.full(E.shape, -1, dtype=np.int64)
    for q in range(len(uvmax)):
        m = spec == q + 1
        edges = uvcrd[off[q]:off[q + 1]]
        cnt = np.searchsorted(edges, E[:, m], side="left")
        out[:, m] = off[q] + cnt - 1
    return out


def near_edge(E, uvcrd, tol):
    """True where an energy lies within `tol` of some mesh edge."""
    idx = np.searchsorted(uvcrd, E)
    lo = uvcrd[np.clip(idx - 1, 0, len(uvcrd) - 1)]
    hi = uvcrd[np.clip(idx, 0, len(uvcrd) - 1)]
    return (np.abs(E - lo) <= tol) | (np.abs(E - hi) <= tol)


def nacl_system(ncell=4, d=2.8, ecdmin=-200.0, K=32, order=6, elecut=11.0):
    """Rock-salt lattice of single-site ions (2*ncell)^3 sites, one Na+ vacancy
    refilled by a Na+ test particle at its lattice site.  Returns
    (params, topo, hist, sitepos, cell, ins_conf, site index)."""
    n = 2 * ncell
    L = n * d
    g = np.arange(n) * d
    z, y, x = np.meshgrid(g, g, g, indexing="ij")
    xyz = np.stack([x.ravel(), y.ravel(), z.ravel()], axis=1)
    ijk = np.stack(np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij"), axis=-1).reshape(-1, 3)
    sign = np.where(ijk.sum(axis=1) % 2 == 0, 1.0, -1.0)   # +1 Na, -1 Cl
    vac = 0                                                  # Na+ site at the origin corner
    keep = np.ones(len(xyz), dtype=bool)
    keep[vac] = False
    na = np.where(keep & (sign > 0))[0]
    cl = np.where(keep & (sign < 0))[0]
    ion = lambda q, nm: S.Species(nm, np.array([q]), np.array([0.0]), np.array([0.0]), np.array([22.99]),
                                  np.zeros((3, 1)))
    topo = S.Topology([ion(1.0, "na"), ion(-1.0, "cl"), ion(1.0, "na_test")],
                      [len(na), len(cl), 1], [A.PT_SOLVENT, A.PT_SOLVENT, A.PT_TEST_FLEX])
    prm = S.default_params(slttype=A.SLT_REFS_FLEX, maxins=1, ms1max=K, splodr=order, elecut=elecut,
                           upljcut=elecut, lwljcut=elecut - 2.0, insposition=A.INSPOS_NOCHANGE,
                           insorient=A.INSROT_NOCHANGE, estype=A.ES_NVT, corrcal=0)
    pos = np.concatenate([xyz[na], xyz[cl]], axis=0) + 0.5 * d   # shift off the box faces
    cell = np.diag([L, L, L]).astype(np.float32)
    ins = (xyz[vac] + 0.5 * d).astype(np.float32)
    return prm, topo, dict(ecdmin=ecdmin), A.as_f32(pos.ravel()), A.as_f32(cell.ravel(order="F")), ins, L


MADELUNG_NACL = 1.747564594633   # NaCl Madelung constant (nearest-neighbour distance convention)
WIGNER_SC = -2.837297479         # Ewald self-image potential constant of a simple cubic lattice
COULOMB = float(np.float32(18.22261721)) ** 2   # e^2/A in kcal/mol as the scaled charges carry it


# Four LJ sites in an 8^3 water box, at these offsets (A) from the box centre; every pair is
# at least 6.5 A apart, and waters are pushed out to 3 A from each, as for the soln workload.
SOLN_SOLUTE_OFFSETS = np.array([[1.5, 0.0, 0.0], [-5.0, 0.0, 0.0], [0.0, 7.0, 0.0], [0.0, 0.0, -10.0]])


def soln_multi_system(seed=11):
    """Solutes in solution (slttype soln) with four solute molecules, for check_mol_configuration:
    (params, topo, hist, sitepos, cell, offsets).  Species: 1 = the LJ sites, 2 = water."""
    nside, box, K = 8, 24.9, 32
    c0 = np.full(3, box / 2)
    centres = c0 + SOLN_SOLUTE_OFFSETS
    wat = S.water_box_frame(nside, box, seed).T.reshape(-1, 3, 3)   # (n, 3 sites, xyz)
    for c in centres:
        for i in range(len(wat)):
            d = wat[i, 0] - c
            d -= box * np.round(d / box)
            r = np.linalg.norm(d)
            if r < 3.0:
                wat[i] += d / max(r, 1e-6) * (3.0 - r)
    topo = S.Topology([S.lj_site(), S.water()], [len(centres), nside ** 3], [A.PT_SOLUTE, A.PT_SOLVENT])
    prm = S.default_params(slttype=A.SLT_SOLN, ms1max=K, maxins=1, corrcal=0, wgtslf=0, hostspec=2)
    pos = np.concatenate([centres, wat.reshape(-1, 3)], axis=0)
    cell = np.diag([box] * 3).astype(np.float32)
    return prm, topo, {}, A.as_f32(pos.ravel()), A.as_f32(cell.ravel(order="F")), SOLN_SOLUTE_OFFSETS


def soln_struct_system(stretch=(1.0, 1.05, 1.3, 1.6), seed=11):
    """Solutes in solution with four water-shaped 3-site solutes whose two O-H bonds are
    stretched by `stretch`, each turned by its own rotation, at SOLN_SOLUTE_OFFSETS in the 8^3
    water box, for check_mol_configuration's structure test: (params, topo, hist, sitepos,
    cell, ideal solute coordinates [3, 3], solute weights)."""
    nside, box, K = 8, 24.9, 32
    c0 = np.full(3, box / 2)
    centres = c0 + SOLN_SOLUTE_OFFSETS
    wat = S.water_box_frame(nside, box, seed).T.reshape(-1, 3, 3)
    for c in centres:
        for i in range(len(wat)):
            d = wat[i, 0] - c
            d -= box * np.round(d / box)
            r = np.linalg.norm(d)
            if r < 3.5:
                wat[i] += d / max(r, 1e-6) * (3.5 - r)
    w = S.water()
    ideal = w.coords.T.copy()                       # O at the origin, H1, H2
    rng = np.random.default_rng(seed + 1)
    slts = []
    for c, s in zip(centres, stretch):
        g = ideal.copy()
        g[1:] *= s
        q = rng.normal(size=4)
        q /= np.linalg.norm(q)
        a, b, cc, d = q
        R = np.array([[a * a + b * b - cc * cc - d * d, 2 * (b * cc - a * d), 2 * (b * d + a * cc)],
                      [2 * (b * cc + a * d), a * a - b * b + cc * cc - d * d, 2 * (cc * d - a * b)],
                      [2 * (b * d - a * cc), 2 * (cc * d + a * b), a * a - b * b - cc * cc + d * d]])
        slts.append((g - g.mean(axis=0)) @ R.T + c)
    solute = S.Species("wshape", w.charge, w.sigma, w.eps, w.mass, w.coords)
    topo = S.Topology([solute, S.water()], [len(centres), nside ** 3], [A.PT_SOLUTE, A.PT_SOLVENT])
    prm = S.default_params(slttype=A.SLT_SOLN, ms1max=K, maxins=1, corrcal=0, wgtslf=0, hostspec=2)
    pos = np.concatenate([np.concatenate(slts, axis=0), wat.reshape(-1, 3)], axis=0)
    cell = np.diag([box] * 3).astype(np.float32)
    return (prm, topo, {}, A.as_f32(pos.ravel()), A.as_f32(cell.ravel(order="F")), ideal,
            np.asarray(w.mass, dtype=np.float64))
