"""Seeded synthetic EPSR systems: molecules, box, r/Q grids and tabulated potentials.

Every array produced here is an INPUT of the hot path (coordinates, potential tables,
transform tables, EP basis); none of it is on the measured path.  Conventions follow the
reference's state layout so that the same arrays can be handed to the reference routines
(for golden vectors) and to the device path:

* coordinates are float32 in box-fraction units, ``x_A / dmax``
  (ato_read_and_save.py:916-960 ``normalise_coordinates``); molecule centre ``xadd`` plus
  per-atom offsets ``xa`` (the absolute position is ``xa + xadd``);
* the r grid follows the float32 recurrence of ``inita`` (epsr_standalone_rev3.py:2945-2998):
  ``x[1]=0``, ``x[2]=0.25*cellst``, ``x[j]=(j-2)*cellst`` built by repeated addition;
  ``xstar = x/dmax`` (``initpt`` epsr_standalone_rev3.py:3749);
* potential tables are 1-based in the grid index: ``tab[pair, iz]`` with ``iz`` in
  ``1..npt`` (index 0 unused), slopes are forward differences on ``xstar``
  (``generate_rp`` epsr_standalone_rev3.py:5845-5864);
* truncation: cosine taper between rminpt and rmaxpt for LJ/EP (``truncate``
  ato_manipulation_rev4.py:693) and the Hummer form for Coulomb (``truncatec`` :715).

Indices in this module are 0-based for molecules, atoms, types and pairs.
"""

from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

f32 = np.float32
COULOMB_KJ = 138.935458  # e^2/(4 pi eps0) in kJ/mol * A
MPZ = 3000  # r-grid capacity of the reference (common/epsr_dimension.py)


# ----------------------------------------------------------------------------- molecules
@dataclass
class MolTemplate:
    name: str
    labels: list          # atom type label per atom
    pos: np.ndarray       # (n,3) float64 Angstrom, relative to the molecule centre
    bonds: list = field(default_factory=list)   # (i, j, length_A) harmonic constraints
    rot_groups: list = field(default_factory=list)  # (axis atom 1, axis atom 2, [rotated atoms]), type ROT


def water_template() -> MolTemplate:
    """Rigid water: O-H 1.0 A, H-O-H 109.47 deg (configuration C1 geometry)."""
    ang = math.radians(109.47) / 2.0
    o = np.zeros(3)
    h1 = np.array([math.sin(ang), 0.0, math.cos(ang)])
    h2 = np.array([-math.sin(ang), 0.0, math.cos(ang)])
    pos = np.stack([o, h1, h2])
    m = np.array([16.0, 1.0, 1.0])
    pos = pos - (m[:, None] * pos).sum(0) / m.sum()
    dhh = float(np.linalg.norm(h1 - h2))
    return MolTemplate("water", ["OW", "HW", "HW"], pos,
                       bonds=[(0, 1, 1.0), (0, 2, 1.0), (1, 2, -dhh)])


def dmso_template() -> MolTemplate:
    """DMSO (C2H6SO): S=O 1.53 A, S-C 1.80 A, C-H 1.09 A, O-S-C 106.7 deg, C-S-C 97.4 deg."""
    cz = math.cos(math.radians(106.7))
    ccs = math.cos(math.radians(97.4))
    b = math.sqrt(((1 - cz * cz) + (ccs - cz * cz)) / 2.0)
    a = math.sqrt(1 - cz * cz - b * b)
    s = np.zeros(3)
    o = np.array([0.0, 0.0, 1.53])
    c1 = 1.80 * np.array([a, b, cz])
    c2 = 1.80 * np.array([-a, b, cz])
    atoms = [s, o, c1, c2]
    labels = ["S", "OD", "C", "C"]
    for c in (c1, c2):
        axis = -c / np.linalg.norm(c)          # C -> S direction
        perp1 = np.cross(axis, [0.0, 0.0, 1.0])
        perp1 /= np.linalg.norm(perp1)
        perp2 = np.cross(axis, perp1)
        th = math.radians(180.0 - 109.5)
        for k in range(3):
            phi = 2 * math.pi * k / 3
            d = -math.cos(th) * axis + math.sin(th) * (math.cos(phi) * perp1 + math.sin(phi) * perp2)
            atoms.append(c + 1.09 * d)
            labels.append("HC")
    pos = np.stack(atoms)
    mass = np.array([32.06, 16.0, 12.01, 12.01] + [1.008] * 6)
    pos = pos - (mass[:, None] * pos).sum(0) / mass.sum()
    bonds = [(0, 1, 1.53), (0, 2, 1.80), (0, 3, 1.80)]
    for ci, h0 in ((2, 4), (3, 7)):
        for k in range(3):
            bonds.append((ci, h0 + k, 1.09))
    # the two methyl groups rotate about their S-C axis (ROT groups, as 200DMSO400Water.ato)
    return MolTemplate("dmso", labels, pos, bonds=bonds, rot_groups=[(0, 2, [4, 5, 6]), (0, 3, [7, 8, 9])])


def atom_template(label: str) -> MolTemplate:
    return MolTemplate(label, [label], np.zeros((1, 3)))


# Per type: charge (e), LJ epsilon (kJ/mol), LJ sigma (A), mass
TYPE_PARAMS = {
    "OW": (-0.8476, 0.65, 3.166, 16.0),
    "HW": (0.4238, 0.0, 0.0, 1.008),
    "S": (0.139, 1.65, 3.56, 32.06),
    "OD": (-0.459, 1.17, 2.93, 16.0),
    "C": (-0.148, 0.276, 3.50, 12.01),
    "HC": (0.09, 0.125, 2.50, 1.008),
    "Si": (2.0, 0.175, 1.0, 28.09),
    "O": (-1.0, 0.65, 3.6, 16.0),
}


def random_rotation(rng: np.random.Generator) -> np.ndarray:
    q = rng.normal(size=4)
    q /= np.linalg.norm(q)
    a, b, c, d = q
    return np.array([
        [a * a + b * b - c * c - d * d, 2 * (b * c - a * d), 2 * (b * d + a * c)],
        [2 * (b * c + a * d), a * a - b * b + c * c - d * d, 2 * (c * d - a * b)],
        [2 * (b * d - a * c), 2 * (c * d + a * b), a * a - b * b - c * c + d * d]])


def _place(rng, L, templates, counts, min_heavy, max_tries=20000):
    """Random centres/orientations, rejecting heavy-atom contacts closer than min_heavy (A)."""
    mols = []
    cell_n = max(1, int(L // max(min_heavy, 1e-3)))
    grid: dict = {}

    def key(p):
        return tuple((np.floor(p / L * cell_n).astype(int)) % cell_n)

    order = []
    for t, n in zip(templates, counts):
        order += [t] * n
    # large molecules first (random order within a type); the box keeps types grouped
    sizes = np.array([len(t.labels) for t in order])
    perm = np.lexsort((rng.permutation(len(order)), -sizes))
    placed = [None] * len(order)
    for idx in perm:
        t = order[idx]
        heavy = [i for i, lab in enumerate(t.labels) if not lab.startswith("H")]
        for _ in range(max_tries):
            centre = rng.uniform(0, L, size=3)
            rot = random_rotation(rng) if len(t.labels) > 1 else np.eye(3)
            pos = centre + t.pos @ rot.T
            ok = True
            for i in heavy:
                p = pos[i] % L
                k = key(p)
                for dx in (-1, 0, 1):
                    for dy in (-1, 0, 1):
                        for dz in (-1, 0, 1):
                            kk = ((k[0] + dx) % cell_n, (k[1] + dy) % cell_n, (k[2] + dz) % cell_n)
                            for q in grid.get(kk, ()):
                                d = p - q
                                d -= L * np.round(d / L)
                                if d @ d < min_heavy * min_heavy:
                                    ok = False
                                    break
                            if not ok:
                                break
                        if not ok:
                            break
                    if not ok:
                        break
                if not ok:
                    break
            if ok:
                for i in heavy:
                    p = pos[i] % L
                    grid.setdefault(key(p), []).append(p)
                placed[idx] = (t, centre, rot)
                break
        else:
            raise RuntimeError("could not place molecule; lower the density or min_heavy")
    return placed


# ----------------------------------------------------------------------------- grids
def make_rgrid(cellst: float, rmaxgr: float, rminpt: float, rmaxpt: float):
    """float32 r grid of ``inita`` (epsr_standalone_rev3.py:2945-2998), 1-based, length npt+1."""
    celstt = f32(cellst)
    x = np.zeros(MPZ + 1, dtype=f32)
    x1dold = f32(-0.5) * celstt
    cellhf = f32(0.25) * celstt
    j = 2
    npt1 = npt2 = nptmin = nptmax = 2
    x1d = x1dold + celstt
    rmaxgr = f32(rmaxgr)
    while j < MPZ and x1d < rmaxgr:
        x[j] = x1d - cellhf
        x1dold = x1d
        cellhf = f32(0.5) * celstt
        if x1d < f32(rminpt):
            nptmin = j + 1
        if x1d < f32(rmaxpt):
            nptmax = j + 1
        if x1d < rmaxgr:
            npt1 = j
        j += 1
        x1d = x1dold + celstt
    x[j] = x1d - cellhf
    npt = j
    npt2 = j - 2
    npt1 = min(npt1, npt2)
    return dict(x=x[: npt + 1].copy(), npt=npt, npt1=npt1, npt2=npt2, nptmin=nptmin, nptmax=nptmax)


def truncate_lj(r, rminpt, rmaxpt):
    """Cosine taper (``truncate`` ato_manipulation_rev4.py:693-712)."""
    w = np.where(r >= rmaxpt, 0.0, np.where(r <= rminpt, 1.0,
                 0.5 * (1.0 + np.cos((r - rminpt) * math.pi / (rmaxpt - rminpt)))))
    return w


def truncate_coul(r, rmaxpt):
    """Hummer charged-cloud taper (``truncatec`` ato_manipulation_rev4.py:715-727)."""
    rat = r / rmaxpt
    w = (1.0 - rat) ** 4 * (1.0 + rat * (1.6 + rat * 0.4))
    return np.where(r >= rmaxpt, 0.0, w)


# ----------------------------------------------------------------------------- system
@dataclass
class System:
    """One periodic box plus everything the hot path reads (0-based molecules/atoms)."""
    name: str
    L: float
    dmax: np.float32
    type_labels: list
    itype: np.ndarray          # (natom,) int32, 0-based type
    mtype: np.ndarray          # (nmol,) int32, 0-based molecule type
    naf: np.ndarray            # (nmol,) int32, first atom (0-based)
    nato: np.ndarray           # (nmol,) int32
    xa: np.ndarray
    ya: np.ndarray
    za: np.ndarray             # (natom,) float32 offsets, box-fraction
    xadd: np.ndarray
    yadd: np.ndarray
    zadd: np.ndarray           # (nmol,) float32 centres, box-fraction
    npairref: np.ndarray       # (ntype,ntype) int32, 0-based pair index
    n1extr: np.ndarray
    n2extr: np.ndarray         # (npairs,) 0-based types of each pair
    cellst: np.float32
    grid: dict
    xstar: np.ndarray          # (npt+1,) float32
    xavs: np.ndarray
    xavs1: np.ndarray
    ecoul: np.ndarray
    ecoul1: np.ndarray         # (npairs, npt+1) float32, iz 1-based
    temperature: float
    simt: np.float32
    nmoltype: int
    moltemplates: list
    bonds: list                # per molecule type: list of (i,j,len_A)
    rminpt: float
    rmaxpt: float
    rmaxgr: float
    charges: np.ndarray        # (ntype,)
    cfrac: np.ndarray          # (ntype,) float32 atom fractions
    meta: dict = field(default_factory=dict)

    @property
    def nmol(self):
        return int(self.mtype.shape[0])

    @property
    def natom(self):
        return int(self.itype.shape[0])

    @property
    def ntype(self):
        return len(self.type_labels)

    @property
    def npairs(self):
        return int(self.n1extr.shape[0])

    @property
    def stepcl(self):
        return f32(self.cellst) / self.dmax


def build_system(name, templates, counts, L, temperature=298.0, cellst=0.03, rminpt=9.0, rmaxpt=12.0,
                 rmaxgr=None, seed=1, min_heavy=2.5, ep_coeffs=0, ep_scale=0.1):
    rng = np.random.default_rng(seed)
    labels = []
    for t in templates:
        for lab in t.labels:
            if lab not in labels:
                labels.append(lab)
    ntype = len(labels)
    npairref = np.zeros((ntype, ntype), dtype=np.int32)
    n1, n2 = [], []
    ip = 0
    for i in range(ntype):
        for j in range(i, ntype):
            npairref[i, j] = npairref[j, i] = ip
            n1.append(i)
            n2.append(j)
            ip += 1
    placed = _place(rng, L, templates, counts, min_heavy)
    dmax = f32(L)
    itype, mtype, naf, nato, offs, centres = [], [], [], [], [], []
    tindex = {t.name: k for k, t in enumerate(templates)}
    a = 0
    for (t, centre, rot) in placed:
        mtype.append(tindex[t.name])
        naf.append(a)
        nato.append(len(t.labels))
        for lab, p in zip(t.labels, t.pos @ rot.T):
            itype.append(labels.index(lab))
            offs.append(p)
        a += len(t.labels)
        c = centre / L
        c = c - np.round(c)      # centres inside [-0.5, 0.5)
        centres.append(c)
    offs = (np.asarray(offs) / float(L)).astype(f32)
    centres = np.asarray(centres).astype(f32)
    if rmaxgr is None:
        rmaxgr = 0.5 * L
    grid = make_rgrid(cellst, rmaxgr, rminpt, rmaxpt)
    x = grid["x"]
    xstar = (x / dmax).astype(f32)
    npt = grid["npt"]
    npairs = len(n1)
    q = np.array([TYPE_PARAMS[lab][0] for lab in labels])
    eps = np.array([TYPE_PARAMS[lab][1] for lab in labels])
    sig = np.array([TYPE_PARAMS[lab][2] for lab in labels])
    r = x.astype(np.float64)
    r[0] = r[1] = max(r[2], 1e-4)
    wlj = truncate_lj(r, rminpt, rmaxpt)
    wc = truncate_coul(r, rmaxpt)
    wlj[npt] = 0.0
    wc[npt] = 0.0
    ecoul = np.zeros((npairs, npt + 1), dtype=f32)
    xavs = np.zeros((npairs, npt + 1), dtype=f32)
    for p in range(npairs):
        i, j = n1[p], n2[p]
        e = math.sqrt(eps[i] * eps[j])
        s = 0.5 * (sig[i] + sig[j])
        lj = np.zeros_like(r)
        if e > 0 and s > 0:
            sr6 = (s / r) ** 6
            lj = 4.0 * e * (sr6 * sr6 - sr6)
        coul = COULOMB_KJ * q[i] * q[j] / r
        tot = np.clip(lj * wlj + coul * wc, -1.0e7, 1.0e7)
        tot[1] = tot[2]
        ecoul[p] = tot.astype(f32)
        if ep_coeffs:
            c = rng.uniform(-ep_scale, ep_scale, size=ep_coeffs)
            sigp = rmaxpt / (ep_coeffs + 2)
            ep = np.zeros_like(r)
            for k in range(ep_coeffs):
                n = k + 2
                xr = r / sigp
                ep += c[k] * np.exp(n * np.log(xr) - xr - math.lgamma(n + 1))
            ep = ep * wlj
            ep[1] = ep[2]
            xavs[p] = ep.astype(f32)
    ecoul1 = slopes(ecoul, xstar, npt)
    xavs1 = slopes(xavs, xstar, npt)
    itype = np.asarray(itype, dtype=np.int32)
    cfrac = np.zeros(ntype, dtype=f32)
    for t in range(ntype):
        cfrac[t] = f32(np.count_nonzero(itype == t)) / f32(itype.shape[0])
    return System(
        name=name, L=float(L), dmax=dmax, type_labels=labels, itype=itype,
        mtype=np.asarray(mtype, dtype=np.int32), naf=np.asarray(naf, dtype=np.int32),
        nato=np.asarray(nato, dtype=np.int32),
        xa=offs[:, 0].copy(), ya=offs[:, 1].copy(), za=offs[:, 2].copy(),
        xadd=centres[:, 0].copy(), yadd=centres[:, 1].copy(), zadd=centres[:, 2].copy(),
        npairref=npairref, n1extr=np.asarray(n1, dtype=np.int32), n2extr=np.asarray(n2, dtype=np.int32),
        cellst=f32(cellst), grid=grid, xstar=xstar, xavs=xavs, xavs1=xavs1, ecoul=ecoul, ecoul1=ecoul1,
        temperature=float(temperature), simt=f32(0.008314) * f32(temperature), nmoltype=len(templates),
        moltemplates=templates, bonds=[t.bonds for t in templates], rminpt=rminpt, rmaxpt=rmaxpt,
        rmaxgr=float(rmaxgr), charges=q, cfrac=cfrac)


def slopes(tab, xstar, npt):
    """Forward-difference slopes on xstar (generate_rp epsr_standalone_rev3.py:5845-5864)."""
    out = np.zeros_like(tab)
    for p in range(tab.shape[0]):
        for j in range(2, npt + 1):
            out[p, j - 1] = (tab[p, j] - tab[p, j - 1]) / (xstar[j] - xstar[j - 1])
        out[p, npt] = f32(0.0)
    return out


# ----------------------------------------------------------------------------- configs
def c1_water(seed=1, nmol=100, rho_atoms=0.1):
    """100 rigid water molecules at 0.1 atoms/A^3 (L = 14.42 A), T = 298 K, EP = 0."""
    L = (3 * nmol / rho_atoms) ** (1.0 / 3.0)
    return build_system("c1_water", [water_template()], [nmol], L, temperature=298.0, seed=seed)


def c2_mixture(seed=1, ndmso=200, nwater=400, rho_atoms=0.1, ep_coeffs=30):
    """200 DMSO + 400 water (3200 atoms) at 0.1 atoms/A^3, T = 298 K, 30-term seeded EP."""
    natom = 10 * ndmso + 3 * nwater
    L = (natom / rho_atoms) ** (1.0 / 3.0)
    return build_system("c2_mixture", [dmso_template(), water_template()], [ndmso, nwater], L,
                        temperature=298.0, seed=seed, ep_coeffs=ep_coeffs, min_heavy=2.0)


def c3_water(seed=1, nmol=20000, rho_atoms=0.1):
    """20,000 water (60,000 atoms, L = 84.3 A), EP on, g(r) bin 0.03 A."""
    L = (3 * nmol / rho_atoms) ** (1.0 / 3.0)
    return build_system("c3_water", [water_template()], [nmol], L, temperature=298.0, seed=seed,
                        ep_coeffs=30, min_heavy=2.5)


def c5_learned(seed=1, ndmso=2700, nwater=5300, rho_atoms=0.1, ep_coeffs=30):
    """Configuration C5: 2,700 DMSO + 5,300 water (8,000 molecules, 42,900 atoms, L = 75.4 A)
    at 0.1 atoms/A^3, T = 298 K, 30-term seeded EP -- the box of the delayed-acceptance runs."""
    natom = 10 * ndmso + 3 * nwater
    L = (natom / rho_atoms) ** (1.0 / 3.0)
    return build_system("c5_learned", [dmso_template(), water_template()], [ndmso, nwater], L,
                        temperature=298.0, seed=seed, ep_coeffs=ep_coeffs, min_heavy=2.0)


def silica(seed=1, natom=300, rho_atoms=0.0662, temperature=1500.0):
    """Amorphous-SiO2-like box of single-atom molecules (Si +2 e / O -1 e)."""
    nsi = natom // 3
    no = natom - nsi
    L = (natom / rho_atoms) ** (1.0 / 3.0)
    return build_system("silica", [atom_template("Si"), atom_template("O")], [nsi, no], L,
                        temperature=temperature, seed=seed, min_heavy=1.4)


def c4_batch(seed=1, nbox=64, amin=300, amax=30000):
    """Configuration C4: ``nbox`` independent boxes whose atom counts are log-uniform in
    [amin, amax] (seeded), alternately rigid water (0.1 atoms/A^3) and SiO2-like single-atom
    boxes (0.0662 atoms/A^3), temperatures uniform in 298-1500 K."""
    rng = np.random.default_rng(seed)
    sizes = np.exp(rng.uniform(math.log(amin), math.log(amax), nbox))
    temps = rng.uniform(298.0, 1500.0, nbox)
    out = []
    for b in range(nbox):
        if b % 2 == 0:
            nmol = max(4, int(round(sizes[b] / 3.0)))
            L = (3 * nmol / 0.1) ** (1.0 / 3.0)
            out.append(build_system("c4_water", [water_template()], [nmol], L, temperature=float(temps[b]),
                                    seed=seed * 1000 + b))
        else:
            out.append(silica(seed=seed * 1000 + b, natom=max(12, int(round(sizes[b]))), temperature=float(temps[b])))
    return out


# ----------------------------------------------------------------------------- transforms
def qgrid(nq, qstep):
    """Q grid of ``inita`` (epsr_standalone_rev3.py:3025-3026): q[i] = qstep*(i-1), 1-based."""
    q = np.zeros(nq + 1, dtype=f32)
    for i in range(1, nq + 1):
        q[i] = f32(qstep) * f32(i - 1)
    return q


def transform_table(sysm: System, q, npt1):
    """A foqols-like sine-integral table F[j, i] (j = r index, i = Q index), 1-based.

    Shaped like ``inita``'s table (epsr_standalone_rev3.py:3045-3071): shell-integrated
    sin(Qr)/Qr weight divided by the uniform-density count ``ycoh[j]``.
    """
    x = sysm.grid["x"].astype(np.float64)
    nq = q.shape[0] - 1
    rho = sysm.natom / sysm.L ** 3
    ycoh = np.zeros(x.shape[0], dtype=f32)
    dr = float(sysm.cellst)
    ycoh[2:npt1 + 1] = (4 * math.pi * rho * x[2:npt1 + 1] ** 2 * dr).astype(f32)
    F = np.zeros((npt1 + 1, nq + 1), dtype=f32)
    qq = q.astype(np.float64)[1:]
    for j in range(2, npt1 + 1):
        qr = qq * x[j]
        sinc = np.where(qr > 0, np.sin(qr) / np.where(qr > 0, qr, 1.0), 1.0)
        g = np.exp(-0.5 * (0.02 * qq * x[j]) ** 2)
        F[j, 1:] = (4 * math.pi * rho * x[j] ** 2 * dr * sinc * g / max(float(ycoh[j]), 1e-30)).astype(f32)
    return F, ycoh


def ep_basis(q, nterms, sigma=0.35, seed=3):
    """A Q-space power-exponential-like EP basis ``expr[(i-1)*nterms + m]`` (1-based flat),
    shaped like ``calc_pwrexpq`` (epsr_standalone_rev3.py:5100-5154)."""
    nq = q.shape[0] - 1
    expr = np.zeros(nq * nterms + 1, dtype=f32)
    for m in range(1, nterms + 1):
        s = sigma * (1.0 + 0.05 * m)
        n = m % 7
        qs = q[1:].astype(np.float64) * s
        alpha = np.arctan(qs)
        with np.errstate(divide="ignore", invalid="ignore"):
            term = np.where(qs > 0, 2 * np.cos(n * alpha) + (1 - qs * qs) * np.sin(n * alpha) / np.where(qs > 0, qs, 1),
                            n + 2.0)
        pn = term / (n + 2.0) / np.sqrt(1 + qs * qs) ** (4 + n)
        expr[1 + (np.arange(nq)) * nterms + (m - 1)] = pn.astype(f32)
    return expr


def pwrexpq_basis(q, nterms, dmin, dstep, sigmab):
    """The Q-space transforms of the power-exponential EP basis functions, shaped and spaced as
    calc_pwrexpq (epsr_standalone_rev3.py:5100-5153, positions from dnext :5312), in double
    precision: ``expr[(i-1)*nterms + m]`` (1-based flat).  The fit of a workload that refines
    its EP uses these, so that the fitted coefficients are those of the r-space basis that
    generate_ep expands."""
    nq = q.shape[0] - 1
    qq = q[1:].astype(np.float64)
    expr = np.zeros(nq * nterms + 1, dtype=f32)
    d, rootd = float(dstep), 1.0
    for m in range(1, nterms + 1):
        sigma = rootd * float(sigmab)
        n = int(d / sigma - 1.0) if (sigma <= d and sigma > 0.0 and m > 1) else 0
        qs = qq * sigma
        alpha = np.arctan(qs)
        with np.errstate(divide="ignore", invalid="ignore"):
            term = np.where(qs > 0, 2.0 * np.cos(n * alpha) + (1.0 - qs * qs) * np.sin(n * alpha) / np.where(
                qs > 0, qs, 1.0), n + 2.0)
        logden = 0.5 * (4 + n) * np.log1p(qs * qs)
        expr[1 + np.arange(nq) * nterms + (m - 1)] = (term / (n + 2.0) * np.exp(-logden)).astype(f32)
        dn, dtest = d + float(dstep), d * float(dmin)
        if dtest > dn:
            dn, rootd = dtest, rootd * math.sqrt(float(dmin))
        d = dn
    return expr


def fit_problem(nq=600, nterms=116, seed=5, noise=0.005):
    """Synthetic fit_expansion inputs: yin = basis . c_true + Gaussian noise (1-based)."""
    rng = np.random.default_rng(seed)
    q = qgrid(nq, 0.05)
    expr = ep_basis(q, nterms)
    c = rng.uniform(-0.05, 0.05, size=nterms)
    E = expr[1:].reshape(nq, nterms).astype(np.float64)
    y = E @ c + rng.normal(0, noise, size=nq)
    yin = np.zeros(nq + 1, dtype=f32)
    yin[1:] = y.astype(f32)
    return dict(q=q, expr=expr, yin=yin, nterms=nterms, npt=nq)


def intra_model(s: System):
    """The intramolecular model of en_atom_intra (molfit.py:923) for system ``s``: the
    templates' harmonic bonds in both atoms' lists (box units; a negative length marks a
    bond-angle pair), per-type masses, unit bond weights x dmax, and the reference potential
    (ecoul) for the non-bonded pairs inside a molecule."""
    natom = int(s.itype.shape[0])
    lists = [[] for _ in range(natom)]
    for m in range(s.nmol):
        a0 = int(s.naf[m])
        for (i, j, length) in s.bonds[int(s.mtype[m])]:
            for (a, b) in ((a0 + i, a0 + j), (a0 + j, a0 + i)):
                lists[a].append((b, f32(length) / f32(s.dmax)))
    mb = max(1, max(len(v) for v in lists))
    iabond = np.full((natom, mb), -1, np.int32)
    tbond = np.zeros((natom, mb), f32)
    for a, v in enumerate(lists):
        for k, (b, t) in enumerate(v):
            iabond[a, k], tbond[a, k] = b, t
    return dict(nbond=np.array([len(v) for v in lists], np.int32), iabond=iabond, tbond=tbond,
                amassa=np.array([TYPE_PARAMS[lab][3] for lab in s.type_labels], f32),
                amassr=np.full(s.npairs, f32(1.0) * f32(s.dmax), f32), xav=s.ecoul, xav1=s.ecoul1,
                stepcl=f32(s.cellst) / f32(s.dmax), simt=f32(s.simt), sizefactor=f32(1.0), tempb=f32(1.0),
                tempang=f32(1.0), refine_intra=False, refine_intra_fac=f32(0.0))


def rotations(s: System):
    """The rotational groups of every molecule of ``s`` from its templates, as the device takes
    them (0-based): ngrot, nrf, nrl per molecule (nrl < nrf: none), axis (groups x 2), first,
    last per group into atoms.  None when no template has groups."""
    if not any(t.rot_groups for t in s.moltemplates):
        return None
    ngrot = np.zeros(s.nmol, np.int32)
    nrf = np.zeros(s.nmol, np.int32)
    nrl = np.full(s.nmol, -1, np.int32)
    axis, first, last, atoms = [], [], [], []
    for m in range(s.nmol):
        groups = s.moltemplates[int(s.mtype[m])].rot_groups
        a0 = int(s.naf[m])
        nrf[m] = len(axis)
        for (i, j, rot) in groups:
            axis.append((a0 + i, a0 + j))
            first.append(len(atoms))
            atoms.extend(a0 + k for k in rot)
            last.append(len(atoms) - 1)
        nrl[m] = len(axis) - 1
        ngrot[m] = len(groups)
    return dict(ngrot=ngrot, nrf=nrf, nrl=nrl, axis=np.array(axis, np.int32).reshape(-1, 2),
                first=np.array(first, np.int32), last=np.array(last, np.int32), atoms=np.array(atoms, np.int32))


# ----------------------------------------------------------------------------- workloads
def intra_energies(s: System, k_bond=1000.0):
    """Per-molecule harmonic bond energies (float32) of the seeded geometry.

    The pair path takes intramolecular energies as an input (they decide whether a
    molecule's first store slot is its own energy, ergpairreference.py:103-118); for a
    synthetic box they are the harmonic deviation of each bond from its template length.
    """
    out = np.zeros(s.nmol, dtype=f32)
    for m in range(s.nmol):
        a0 = int(s.naf[m])
        e = 0.0
        for (i, j, length) in s.bonds[int(s.mtype[m])]:
            d = np.array([s.xa[a0 + i] - s.xa[a0 + j], s.ya[a0 + i] - s.ya[a0 + j], s.za[a0 + i] - s.za[a0 + j]],
                         dtype=np.float64) * float(s.dmax)
            e += k_bond * (float(np.sqrt(d @ d)) - abs(length)) ** 2
        out[m] = f32(e)
    return out


@dataclass
class EpRefinement:
    """The potential-refinement state of potential_par that ptgnsq and generate_ep read
    (epsr_standalone_rev3.py:3946-3962, :5876-6022): one coefficient set per atom pair
    (irefpcof(ip) = ip), the r-space Poisson basis parameters of the reference's defaults
    (pdstep 0.1, pdmin 1 + pdstep/rminpt, pdmax rmaxpt), the truncation wfac and the
    amplitude controls."""
    pcoefp: np.ndarray       # (nsets, nterms+1) [set, ic]: ic = 1 the amplitude, 2.. the terms
    iref: np.ndarray         # (npairs,) 0-based set of each pair
    efacp: np.ndarray        # (nsets,)
    wfac: np.ndarray         # (npt+1,) truncate(r, rminpt, rmaxpt), 0 at npt
    pdmin: float
    pdstep: float
    pdmax: float
    psigma2: float
    rho: float
    rbroad: float = 0.0
    potfac: float = 0.2
    absolute_energy: float = 10.0
    erequnit: float = 1.0
    ereqstep: float = 0.0
    potfacamp: float = 0.5


def ep_refinement(s, nterms, seed=7):
    """Seeded potential-refinement state for system ``s`` (an EPSR run in progress: unit
    amplitudes and small nonzero coefficients)."""
    rng = np.random.default_rng(seed)
    npairs = s.npairs
    pc = np.zeros((npairs, nterms + 1), dtype=f32)
    pc[:, 1] = 1.0
    pc[:, 2:] = (rng.standard_normal((npairs, nterms - 1)) * 0.02).astype(f32)
    npt = s.grid["npt"]
    wfac = truncate_lj(s.grid["x"].astype(np.float64), s.rminpt, s.rmaxpt).astype(f32)
    wfac[npt] = 0.0
    pdstep = f32(0.1)
    return EpRefinement(pcoefp=pc, iref=np.arange(npairs, dtype=np.int32), efacp=np.ones(npairs, f32), wfac=wfac,
                        pdmin=float(f32(1.0) + pdstep / f32(s.rminpt)), pdstep=float(pdstep), pdmax=float(s.rmaxpt),
                        psigma2=0.01, rho=float(f32(0.1)))


@dataclass
class Workload:
    """One EPSR iteration's inputs for the pair path on a box."""
    name: str
    system: System
    eintra: np.ndarray
    q: np.ndarray            # (nq+1,) 1-based
    foqols: np.ndarray       # (npt1+1, nq+1): F[j, i] (Q index fastest)
    ycoh: np.ndarray         # (npt+1,)
    expr: np.ndarray         # (nq*nterms+1,) 1-based flat, row-major by Q
    nterms: int
    data: np.ndarray         # (ndata, nq+1) synthetic interference functions
    weights: np.ndarray      # (ndata, npairs) float64 pair weights of each dataset (real*8 cwt)
    wholerot: np.ndarray
    wholetrans: np.ndarray
    ntimes: int = 5
    nmolcell: int = 10
    rejrate: float = 0.75
    ngrsamples: int = 0
    xwt: np.ndarray = None   # (npairs,) stog offsets
    ep: EpRefinement = None  # potential refinement after the fits (None: the EP stays fixed)
    intra: int = 0           # molfit cycles between intramolecular cycles (0: rigid molecules, none)
    stepmi: float = 1.0      # intramolecular step flag (> 0 moves the atoms of multi-atom molecules)
    data_source: str = "analytic"   # where the data sets come from
    rotfreq: int = 0         # internal rotations of the templates' ROT groups every rotfreq cycles (0: none)
    internrot: np.ndarray = None    # (nmoltype,) starting internal-rotation step (fraction of pi)

    @property
    def nq(self):
        return int(self.q.shape[0] - 1)


def make_workload(name="c2_mixture", seed=1, nq=None, qstep=0.05, nterms=116, ndata=None, ntimes=5, refine=True,
                  intra=0, data_source="auto", rotfreq=0):
    """One iteration's inputs on a named configuration, 5 MC sweeps per iteration and a
    116-term Poisson-like EP basis.  C2 (c2_mixture): 200 DMSO + 400 water, three isotope
    data sets (deuterated, protiated, 50:50), Q to 30 A^-1 (600 points).  C3 (c3_water):
    20,000 water, one data set, Q to 50 A^-1 (1,000 points).  C1 (c1_water): 100 water.
    ``refine``: each iteration also refines the EP from the fits (ptgnsq's coefficient
    increment and generate_ep), as the reference does while its potential factor is on.
    ``intra`` > 0: flexible molecules -- every intra-th molfit cycle is an intramolecular one
    (the templates' bonds and bond-angle pairs, intra_model), as molfit's nisum counter picks."""
    if nq is None:
        nq = 1000 if name == "c3_water" else 600
    if ndata is None:
        ndata = 1 if name == "c3_water" else 3
    if name == "c2_mixture":
        s = c2_mixture(seed=seed)
    elif name == "c1_water":
        s = c1_water(seed=seed)
    elif name == "c3_water":
        s = c3_water(seed=seed)
    else:
        raise ValueError(name)
    rng = np.random.default_rng(seed + 100)
    q = qgrid(nq, qstep)
    npt1 = s.grid["npt1"]
    F, ycoh = transform_table(s, q, npt1)
    ep = ep_refinement(s, nterms) if refine else None
    expr = pwrexpq_basis(q, nterms, ep.pdmin, ep.pdstep, ep.psigma2) if refine else ep_basis(q, nterms)
    w = rng.uniform(0.2, 1.0, size=(ndata, s.npairs))
    w /= w.sum(axis=1, keepdims=True)
    data = np.zeros((ndata, nq + 1), dtype=f32)
    qq = q.astype(np.float64)
    for d in range(ndata):
        data[d, 1:] = (0.05 * np.sin(2.9 * qq[1:] + d) * np.exp(-0.05 * qq[1:])
                       + rng.normal(0, 0.005, size=nq)).astype(f32)
    # the data sets the method produced under a perturbed potential (synthdata.py), when they
    # have been generated for this box and Q grid; otherwise the analytic stand-in above
    src = "analytic"
    if data_source == "auto" and seed == 1:
        from . import synthdata
        got = synthdata.load(name)
        if got is not None and got[1].shape[1] == nq + 1 and got[0].shape[1] == s.npairs:
            w, data = got
            src = "method under a perturbed potential (synthdata.py)"
    nmt = s.nmoltype
    wholerot = np.full(nmt, f32(10.0 / 180.0), dtype=f32)
    wholetrans = np.full(nmt, f32(0.5) / s.dmax, dtype=f32)
    xwt = np.linspace(0.5, 1.5, s.npairs).astype(f32)
    return Workload(name=name, system=s, eintra=intra_energies(s), q=q, foqols=F, ycoh=ycoh, expr=expr,
                    nterms=nterms, data=data, weights=w, wholerot=wholerot, wholetrans=wholetrans, ntimes=ntimes,
                    xwt=xwt, ep=ep, intra=int(intra), data_source=src,
                    rotfreq=int(rotfreq) if rotations(s) is not None else 0,
                    internrot=np.array([f32(0.05) if t.rot_groups else f32(0.0) for t in s.moltemplates], f32))
