"""Synthetic solution / reference systems and the setparam-equivalent topology.

No MD trajectory ships with the reference and there is no network, so the
workloads are seeded synthetic systems with the shapes the benchmark
configurations describe: rigid 3-site water on a cubic lattice with random
orientations and Gaussian centre-of-mass jitter, plus the solutes (a single
LJ site, a benzene-like 12-site ring, random-walk chains).

`Topology` reproduces what setparam (erdst/setconf.F90:516-844) derives
from MDinfo / MolPrmN / SltInfo: molecule order, LJ type tables with the
arithmetic-sigma / geometric-epsilon rule (setconf.F90:756-826), charges
scaled by 18.22261721 (setconf.F90:834) and the solvent-species numbering
uvspec (erdst/engproc.F90:112-118).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _capi as A

CHARGE_SCALE = np.float32(18.22261721)      # setconf.F90:834
KB_KCAL = 8.314510e-3 / 4.184                # setconf.F90:304 (kcal/mol/K)

MASS = {"O": 15.9994, "H": 1.00794, "C": 12.0107, "X": 39.948}


@dataclass
class Species:
    """One molecule type: per-site charge (e), sigma (A), epsilon (kcal/mol), mass."""
    name: str
    charge: np.ndarray
    sigma: np.ndarray
    eps: np.ndarray
    mass: np.ndarray
    coords: np.ndarray | None = None    # body-fixed coordinates (3, n) for rigid solutes

    @property
    def nsite(self) -> int:
        return len(self.charge)


def water() -> Species:
    """TIP3P-like rigid water: O q=-0.834 sigma=3.1506 eps=0.1521, H q=+0.417."""
    th = np.deg2rad(104.52) / 2.0
    r = 0.9572
    xyz = np.array([[0.0, 0.0, 0.0],
                    [r * np.sin(th), r * np.cos(th), 0.0],
                    [-r * np.sin(th), r * np.cos(th), 0.0]]).T
    return Species("water", np.array([-0.834, 0.417, 0.417]), np.array([3.1506, 0.0, 0.0]),
                   np.array([0.1521, 0.0, 0.0]), np.array([MASS["O"], MASS["H"], MASS["H"]]), xyz)


def lj_site(sigma=3.73, eps=0.294) -> Species:
    return Species("ljsite", np.zeros(1), np.array([sigma]), np.array([eps]), np.array([MASS["X"]]),
                   np.zeros((3, 1)))


def benzene_ring() -> Species:
    """12-site ring: C-C 1.40 A, C-H 1.08 A; C q=-0.115 sigma=3.55 eps=0.07, H q=+0.115 sigma=2.42 eps=0.03."""
    xyz, q, sg, ep, ms = [], [], [], [], []
    for k in range(6):
        a = np.pi / 3.0 * k
        xyz.append([1.40 * np.cos(a), 1.40 * np.sin(a), 0.0])
        q.append(-0.115); sg.append(3.55); ep.append(0.07); ms.append(MASS["C"])
    for k in range(6):
        a = np.pi / 3.0 * k
        xyz.append([2.48 * np.cos(a), 2.48 * np.sin(a), 0.0])
        q.append(0.115); sg.append(2.42); ep.append(0.03); ms.append(MASS["H"])
    return Species("ring12", np.array(q), np.array(sg), np.array(ep), np.array(ms), np.array(xyz).T)


def random_chain(nsite: int, seed: int, step=1.5, qsd=0.3, sigma=(2.5, 3.8), eps=(0.03, 0.2)) -> Species:
    """Seeded random walk with `step` A bonds, charges N(0,qsd) shifted to net zero."""
    rng = np.random.default_rng(seed)
    xyz = np.zeros((nsite, 3))
    for i in range(1, nsite):
        for _ in range(100):
            d = rng.normal(size=3)
            d *= step / np.linalg.norm(d)
            cand = xyz[i - 1] + d
            if i < 2 or np.min(np.linalg.norm(xyz[:i - 1] - cand, axis=1)) > 0.95 * step:
                break
        xyz[i] = cand
    q = rng.normal(0.0, qsd, size=nsite)
    q -= q.mean()
    sg = rng.uniform(sigma[0], sigma[1], size=nsite)
    ep = rng.uniform(eps[0], eps[1], size=nsite)
    ms = np.full(nsite, MASS["C"])
    return Species(f"chain{nsite}", q, sg, ep, ms, (xyz - xyz.mean(axis=0)).T)


def ring_recipe_solute(nsite: int, seed: int) -> Species:
    """Rigid solute built from the ring's site types: a seeded 1.40 A random walk
    whose sites alternate C-like / H-like parameters (net charge zero for even n)."""
    rng = np.random.default_rng(seed)
    xyz = np.zeros((nsite, 3))
    for i in range(1, nsite):
        for _ in range(200):
            d = rng.normal(size=3)
            d *= 1.40 / np.linalg.norm(d)
            cand = xyz[i - 1] + d
            if i < 2 or np.min(np.linalg.norm(xyz[:i - 1] - cand, axis=1)) > 1.3:
                break
        xyz[i] = cand
    q = np.where(np.arange(nsite) % 2 == 0, -0.115, 0.115)
    if nsite % 2 == 1:
        q[-1] = 0.0
    sg = np.where(np.arange(nsite) % 2 == 0, 3.55, 2.42)
    ep = np.where(np.arange(nsite) % 2 == 0, 0.07, 0.03)
    ms = np.where(np.arange(nsite) % 2 == 0, MASS["C"], MASS["H"])
    return Species(f"ringrecipe{nsite}", q, sg, ep, ms, (xyz - xyz.mean(axis=0)).T)


def _rot_from_quat(q):
    w, x, y, z = q
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y)],
                     [2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x)],
                     [2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)]])


def random_packing(n: int, box: float, rng, dmin: float = 2.5, max_tries: int = 5000, obstacle=None,
                   obstacle_r: float = 0.0):
    """n points in a periodic cube by random sequential addition with a minimum
    separation `dmin` (and at least `obstacle_r` from the point, or every row of the
    points, `obstacle`): a disordered packing with the density fluctuations and cavities
    of a liquid (the lattice has none)."""
    if obstacle is not None:
        obstacle = np.atleast_2d(np.asarray(obstacle, dtype=np.float64))
    nc = max(1, int(box // dmin))
    h = box / nc
    cells = {}
    pts = np.empty((n, 3))
    k = 0
    while k < n:
        for _ in range(max_tries):
            p = rng.uniform(0.0, box, 3)
            if obstacle is not None:
                d = p - obstacle
                d -= box * np.round(d / box)
                if np.einsum("ij,ij->i", d, d).min() < obstacle_r * obstacle_r:
                    continue
            c = tuple((p // h).astype(int) % nc)
            ok = True
            for dz in (-1, 0, 1):
                for dy in (-1, 0, 1):
                    for dx in (-1, 0, 1):
                        for j in cells.get(((c[0] + dx) % nc, (c[1] + dy) % nc, (c[2] + dz) % nc), ()):
                            d = pts[j] - p
                            d -= box * np.round(d / box)
                            if d @ d < dmin * dmin:
                                ok = False
                                break
                        if not ok:
                            break
                    if not ok:
                        break
                if not ok:
                    break
            if ok:
                pts[k] = p
                cells.setdefault(c, []).append(k)
                k += 1
                break
        else:
            raise RuntimeError("random packing: too dense for the minimum separation")
    return pts


def water_box_frame(nside: int, box: float, seed: int, jitter=0.3, avoid=None, avoid_r=3.0, packing="lattice"):
    """Coordinates (3, 3*nside^3) of nside^3 waters with random orientations.

    packing "lattice": centres of mass on the n^3 lattice plus Gaussian
    `jitter`; "random": a random sequential packing at the same density.
    `avoid`: optional point (or rows of points); water oxygens closer than `avoid_r`
    to it are pushed radially out to `avoid_r` (keeps a soln solute out of the hard
    core).  With several points the random packing keeps every oxygen `avoid_r` away
    from all of them; the lattice packing pushes from the nearest one.
    """
    rng = np.random.default_rng(seed)
    wat = water()
    com_body = (wat.coords * wat.mass).sum(axis=1) / wat.mass.sum()
    body = wat.coords - com_body[:, None]
    n = nside ** 3
    if packing == "random":
        com = random_packing(n, box, rng, obstacle=None if avoid is None else np.asarray(avoid, dtype=np.float64),
                             obstacle_r=avoid_r)
    else:
        g = (np.arange(nside) + 0.5) * (box / nside)
        cz, cy, cx = np.meshgrid(g, g, g, indexing="ij")
        com = np.stack([cx.ravel(), cy.ravel(), cz.ravel()], axis=1) + rng.normal(0.0, jitter, size=(n, 3))
    q = rng.normal(size=(n, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    out = np.empty((n, 3, 3))
    for i in range(n):
        out[i] = (_rot_from_quat(q[i]) @ body).T + com[i]
    if avoid is not None:
        avoid = np.atleast_2d(np.asarray(avoid, dtype=np.float64))
        for i in range(n):
            d = out[i, 0] - avoid
            d -= box * np.round(d / box)
            rr = np.linalg.norm(d, axis=1)
            j = int(np.argmin(rr))
            r = rr[j]
            if r < avoid_r:
                shift = d[j] / max(r, 1e-6) * (avoid_r - r)
                out[i] += shift
    return out.reshape(-1, 3).T


@dataclass
class Topology:
    """setparam's view of a system: molecule list and interaction tables."""
    species: list               # [Species], in MDinfo order
    counts: list                # molecules per species
    kinds: list                 # PT_* per species
    numsite: np.ndarray = field(init=False)
    sluvid: np.ndarray = field(init=False)
    uvspec: np.ndarray = field(init=False)
    charge: np.ndarray = field(init=False)
    ljtype: np.ndarray = field(init=False)
    sitemass: np.ndarray = field(init=False)
    ljtype_max: int = field(init=False)
    ljene_mat: np.ndarray = field(init=False)
    ljlensq_mat: np.ndarray = field(init=False)
    bfcoord: np.ndarray | None = field(init=False)
    numslv: int = field(init=False)

    def __post_init__(self):
        numsite, sluvid, moltype = [], [], []
        for t, (sp, cnt, kind) in enumerate(zip(self.species, self.counts, self.kinds)):
            numsite += [sp.nsite] * cnt
            sluvid += [kind] * cnt
            moltype += [t + 1] * cnt
        self.numsite = A.as_i32(numsite)
        self.sluvid = A.as_i32(sluvid)
        moltype = np.array(moltype, dtype=np.int32)
        # uvspec (engproc.F90:112-118)
        slt_types = {moltype[i] for i in range(len(moltype)) if self.sluvid[i] > 0}
        numslt = int((self.sluvid > 0).sum())
        uv = moltype.copy()
        if numslt == 1:
            st = slt_types.pop()
            uv[self.sluvid != 0] = 0
            uv[(self.sluvid == 0) & (moltype > st)] -= 1
            self.numslv = len(self.species) - 1
        else:
            self.numslv = len(self.species)
        self.uvspec = A.as_i32(uv)
        # LJ types (setconf.F90:756-777) and mixing (setconf.F90:813-826)
        table = []
        ljtype, charge, mass = [], [], []
        for sp, cnt in zip(self.species, self.counts):
            tt = []
            for s in range(sp.nsite):
                key = (np.float32(sp.sigma[s]), np.float32(sp.eps[s]))
                if key not in table:
                    table.append(key)
                tt.append(table.index(key) + 1)
            ljtype += tt * cnt
            charge += list(sp.charge) * cnt
            mass += list(sp.mass) * cnt
        self.ljtype = A.as_i32(ljtype)
        self.charge = (CHARGE_SCALE * np.asarray(charge, dtype=np.float32)).astype(np.float32)
        self.sitemass = A.as_f32(mass)
        n = len(table)
        self.ljtype_max = n
        sg = np.array([t[0] for t in table], dtype=np.float32)
        ep = np.array([t[1] for t in table], dtype=np.float32)
        lensq = np.empty((n, n), dtype=np.float32)
        ene = np.empty((n, n), dtype=np.float32)
        for i in range(n):
            lensq[:, i] = ((sg + sg[i]) / np.float32(2.0)) ** 2
            ene[:, i] = np.sqrt(ep * ep[i])
        self.ljlensq_mat = np.asfortranarray(lensq).ravel(order="F").astype(np.float32)
        self.ljene_mat = np.asfortranarray(ene).ravel(order="F").astype(np.float32)
        self.bfcoord = None
        for sp, kind in zip(self.species, self.kinds):
            if kind == A.PT_TEST_RIGID or kind == A.PT_TEST_FLEX:
                self.bfcoord = A.as_f32(np.asarray(sp.coords, dtype=np.float64).T.ravel())

    @property
    def nummol(self) -> int:
        return len(self.numsite)

    def as_struct(self):
        keep = []

        def p(a, t):
            if a is None:
                return None
            keep.append(a)
            return A.ptr(a, t)

        s = A.ErmodTopology(
            nummol=self.nummol, numsite=p(self.numsite, C.c_int32), sluvid=p(self.sluvid, C.c_int32),
            uvspec=p(self.uvspec, C.c_int32), charge=p(self.charge, C.c_float),
            ljtype=p(self.ljtype, C.c_int32), sitemass=p(self.sitemass, C.c_float),
            ljtype_max=self.ljtype_max, ljene_mat=p(self.ljene_mat, C.c_float),
            ljlensq_mat=p(self.ljlensq_mat, C.c_float), bfcoord=p(self.bfcoord, C.c_float))
        return s, keep


DEFAULT_HIST = dict(eclbin=5.0e-2, ecfbin=2.0e-3, ec0bin=2.0e-4, finfac=10.0, ecdmin=-20.0,
                    ecfmns=-0.20, ecdcen=0.0, eccore=20.0, ecdmax=1.0e11, pecore=200)


def default_params(**kw) -> dict:
    """&ene_param after iniparam's defaults (setconf.F90:174-262) for these workloads."""
    p = dict(slttype=A.SLT_REFS_RIGID, boxshp=A.SYS_PERIODIC, estype=A.ES_NPT, cltype=A.EL_PME,
             ljswitch=A.LJSWT_POT_CHM, splodr=4, ms1max=64, ms2max=64, ms3max=64, maxins=1000,
             corrcal=1, selfcal=0, wgtslf=1, insposition=A.INSPOS_RANDOM, insorient=A.INSROT_RANDOM,
             iseed=123456789, temp=300.0 * KB_KCAL, elecut=12.0, lwljcut=10.0, upljcut=12.0, screen=0.35,
             ins_chunk=0, ecorr_batch=0, weight_bits=0, proposal=A.PROPOSAL_UNIFORM,
             keep_uvengy=0, ecorr_path=0, spectrum_path=0, graph_mode=0, stage_timing=0,
             lwreg=0.0, upreg=0.0, hostspec=0, insstructure=0, lwstr=0.0, upstr=0.0)
    p.update(kw)
    for k in ("ms2max", "ms3max"):
        if k not in kw:
            p[k] = p["ms1max"]
    return p


def params_struct(p: dict) -> A.ErmodParams:
    s = A.ErmodParams()
    for k, v in p.items():
        setattr(s, k, v)
    return s


def hist_struct(h: dict | None = None) -> A.ErmodHist:
    hh = dict(DEFAULT_HIST)
    if h:
        hh.update(h)
    return A.ErmodHist(**hh)


@dataclass
class Workload:
    """A complete synthetic run: parameters, topology, mesh settings and frames."""
    name: str
    params: dict
    topo: Topology
    hist: dict
    box: float
    nside: int
    nframes: int
    seed: int
    solute_center: np.ndarray | None = None     # soln: fixed solute position
    packing: str = "lattice"                     # water centres: "lattice" + jitter or "random"
    avoid_sites: bool = False                    # soln: keep waters avoid_r from every solute site
    avoid_r: float = 3.0

    def frame(self, i: int):
        """sitepos (3*numatm_phys float32, Fortran order) and cell (9 float32) of frame i."""
        avoid = self.solute_center
        if self.avoid_sites and self.solute_center is not None:
            avoid = np.concatenate([(np.asarray(sp.coords) + self.solute_center[:, None]).T
                                    for sp, kind in zip(self.topo.species, self.topo.kinds) if kind == A.PT_SOLUTE])
        wat = water_box_frame(self.nside, self.box, self.seed * 1000003 + i, avoid=avoid, avoid_r=self.avoid_r,
                              packing=self.packing)
        parts = []
        for sp, cnt, kind in zip(self.topo.species, self.topo.counts, self.topo.kinds):
            if kind == A.PT_SOLVENT and sp.name == "water":
                parts.append(wat)
            elif kind == A.PT_SOLUTE:
                parts.append(np.asarray(sp.coords) + self.solute_center[:, None])
        pos = np.concatenate(parts, axis=1)
        cell = np.diag([self.box] * 3).astype(np.float32)
        return A.as_f32(pos.T.ravel()), A.as_f32(cell.ravel(order="F"))


def make_workload(config: int, small: bool = False, maxins: int | None = None, seed: int = 7) -> Workload:
    """Configurations 1..5 (soln LJ site, refs ring, precision chain, batching, learned).

    `small` shrinks the system (for CPU-oracle parity tests) while keeping its recipe.
    """
    if config == 1:
        nside, box, K = (10, 31.04, 32)
        if small:
            nside, box, K = 8, 24.9, 32
        sp = [lj_site(), water()]
        topo = Topology(sp, [1, nside ** 3], [A.PT_SOLUTE, A.PT_SOLVENT])
        prm = default_params(slttype=A.SLT_SOLN, ms1max=K, maxins=1, corrcal=0, wgtslf=0)
        return Workload("soln-ljsite-water1000", prm, topo, {}, box, nside, 10, seed,
                        solute_center=np.array([box / 2] * 3))
    if config in (2, 4, 5):
        nside, box, K = 16, 49.6, 64
        mi = {2: 2000, 4: 500, 5: 100000}[config]
        if small:
            nside, box, K = 8, 24.9, 32
            mi = 64
        if maxins is not None:
            mi = maxins
        slt = benzene_ring() if config == 2 else ring_recipe_solute(200 if config == 5 else 64, seed)
        topo = Topology([water(), slt], [nside ** 3, 1], [A.PT_SOLVENT, A.PT_TEST_RIGID])
        prm = default_params(ms1max=K, maxins=mi)
        nfr = {2: 20, 4: 20, 5: 50}[config]
        return Workload({2: "refs-ring12-water4096", 4: "batch-solutes-water4096",
                         5: "learned-200site-water4096"}[config], prm, topo, {}, box, nside, nfr, seed)
    if config == 3:
        nside, box, K, mi = 32, 99.3, 128, 4096
        if small:
            nside, box, K, mi = 8, 24.9, 32, 64
        if maxins is not None:
            mi = maxins
        slt = random_chain(60, seed)
        topo = Topology([water(), slt], [nside ** 3, 1], [A.PT_SOLVENT, A.PT_TEST_RIGID])
        prm = default_params(ms1max=K, maxins=mi)
        return Workload("precision-chain60-water32768", prm, topo, dict(ecdmin=-80.0), box, nside, 10, seed)
    raise ValueError(config)


def make_batch_workloads(nsolutes: int = 64, small: bool = False, maxins=None, seed: int = 7,
                         site_range=(10, 300)) -> list[Workload]:
    """Configuration 4: `nsolutes` rigid solutes of seeded sizes U[site_range] built with the ring
    recipe, each with its own insertion stream, all sharing the configuration-2 water box and frames.
    `maxins` may be an int or one count per solute."""
    rng = np.random.default_rng(seed + 404)
    sizes = rng.integers(site_range[0], site_range[1] + 1, size=nsolutes)
    base = make_workload(4, small=small, seed=seed)
    counts = [maxins] * nsolutes if maxins is None or np.isscalar(maxins) else list(maxins)
    out = []
    for j, n in enumerate(sizes):
        slt = ring_recipe_solute(int(n), seed * 7919 + j)
        topo = Topology([water(), slt], [base.nside ** 3, 1], [A.PT_SOLVENT, A.PT_TEST_RIGID])
        prm = dict(base.params, iseed=int(base.params["iseed"]) + j)
        if counts[j] is not None:
            prm["maxins"] = int(counts[j])
        out.append(Workload(f"batch{j}-s{int(n)}", prm, topo, {}, base.box, base.nside, base.nframes, seed))
    return out
