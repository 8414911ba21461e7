"""Load a synthetic System into the reference's COMMON-block modules (golden generation only).

Used by ``make_golden.py`` in a container where the reference translation is importable;
it writes the same arrays the reference's own setup (``inita``/``initpt``/``minitc``)
would leave behind, restricted to what the hot-path routines read:

* molfit.py:52-541 (whole-molecule branch), en_change :806-919, en_atom_inter_scale
  :1251-1279, en_mole_pair :1528-1578, en_mole_intra :1327 / en_atom_intra :923;
* cellneighbourlist.py:23-183, ergpairreference.py:63-210, fmolec1
  ato_manipulation_rev4.py:2374-2528, atogen :3640-3899;
* gensq epsr_standalone_rev3.py:4731, stog ato_manipulation_rev4.py:4067,
  fit_expansion epsr_standalone_rev3.py:4806.
"""

from __future__ import annotations

import numpy as np

f32 = np.float32


def reference_root():
    """The checkout of the reference (its top directory, holding src/epsr26), from the
    environment variable EPSR_REFERENCE.  Only the fixture generators read it."""
    import os
    root = os.environ.get("EPSR_REFERENCE")
    if not root or not os.path.isdir(os.path.join(root, "src", "epsr26")):
        raise SystemExit("set EPSR_REFERENCE to the reference checkout (the directory holding src/epsr26)")
    return root


def load_reference(src=None):
    import os
    import sys
    if src is None:
        src = os.path.join(reference_root(), "src")
    os.environ.setdefault("PYTHONDONTWRITEBYTECODE", "1")
    sys.dont_write_bytecode = True
    if src not in sys.path:
        sys.path.insert(0, src)
    import epsr26  # noqa: F401
    from epsr26 import common
    from epsr26.programs import load
    ep = load("epsr")
    return common, ep


def populate(sysm, *, stepr=1.0, stepm=0.5, rejrate=0.75, wholerot=None, wholetrans=None):
    """Fill the reference COMMON modules from ``sysm`` (configs.System).

    stepr/stepm are the input step flags (>0 enables whole-molecule rotation/translation);
    wholerot/wholetrans are per-molecule-type step sizes (box units for translation,
    fraction of pi for rotation).  Returns nothing.
    """
    from epsr26 import common
    from epsr26.common import (cellneighbourlist, clustercom, epsr16, ergpairreference, lattice, molecom,
                               molecom_mod, potential_par, ran1com)
    from epsr26.common import coordconstraints_mod, threebody_mod, containerforces_mod

    common.reset()
    nmol, natom, ntype, npairs = sysm.nmol, sysm.natom, sysm.ntype, sysm.npairs
    dmax = sysm.dmax
    # lattice (cubic box, already normalised by dmax)
    lattice.cubic = True
    lattice.alat = lattice.blat = lattice.clat = f32(1.0)
    lattice.alatx = lattice.blaty = lattice.clatz = f32(1.0)
    lattice.blatx = lattice.clatx = lattice.claty = f32(0.0)
    for v in (lattice.alatc, lattice.blatc, lattice.clatc):
        v[:] = 0.0
    lattice.alatc[1] = lattice.blatc[2] = lattice.clatc[3] = f32(1.0)
    clustercom.dmax = dmax
    clustercom.volume = f32(1.0)
    clustercom.nmol = nmol
    clustercom.nmoltype = sysm.nmoltype
    molecom.natom = natom
    molecom.natomr = natom
    molecom.ntype = ntype
    molecom.npairs = npairs
    molecom.dmaxmol = dmax
    molecom.sizefactor = f32(1.0)
    molecom.simt = sysm.simt
    molecom.simtk = f32(sysm.temperature)
    molecom.stepr = f32(stepr)
    molecom.stepm = f32(stepm)
    molecom.stepri = f32(0.0)
    molecom.stepmi = f32(0.0)
    molecom.tolout = f32(0.0)
    molecom.tempb = f32(1.0)
    molecom.tempang = f32(1.0)
    molecom.tempangwt = f32(1.0)
    molecom.tempangreq = f32(1.0)
    molecom.tempdih = f32(0.0)
    molecom.tempdihwt = f32(0.0)
    molecom.tempdihreq = f32(0.0)
    molecom.refine_intra = False
    for t in range(ntype):
        molecom.cfrac[t + 1] = sysm.cfrac[t]
    for t1 in range(ntype):
        for t2 in range(ntype):
            molecom.npairref[t1 + 1, t2 + 1] = sysm.npairref[t1, t2] + 1
    for p in range(npairs):
        molecom.n1extr[p + 1] = sysm.n1extr[p] + 1
        molecom.n2extr[p + 1] = sysm.n2extr[p] + 1
        molecom.amassr[p + 1] = f32(1.0) * dmax
        potential_par.irefpcof[p + 1] = p + 1
        potential_par.rminex[p + 1] = f32(-2.0)
    molecom_mod.coarsegraining = False
    molecom_mod.natomsphere = np.ones(41, dtype=np.float32)
    for m in range(nmol):
        im = m + 1
        naf = int(sysm.naf[m]) + 1
        nato = int(sysm.nato[m])
        clustercom.naf[im] = naf
        clustercom.nal[im] = naf + nato - 1
        clustercom.nato[im] = nato
        clustercom.mtype[im] = int(sysm.mtype[m]) + 1
        clustercom.ngrot[im] = 0
        clustercom.nrf[im] = 0
        clustercom.nrl[im] = 0
        clustercom.tethered[im] = False
        clustercom.xadd[im] = sysm.xadd[m]
        clustercom.yadd[im] = sysm.yadd[m]
        clustercom.zadd[im] = sysm.zadd[m]
        # bonds of this molecule type (harmonic intra energy; en_atom_intra molfit.py:923)
        for (i, j, length) in sysm.bonds[int(sysm.mtype[m])]:
            ia = naf + i
            ja = naf + j
            for (a, b) in ((ia, ja), (ja, ia)):
                molecom.nbond[a] += 1
                molecom.iabond[a, molecom.nbond[a]] = b
                molecom.tbond[a, molecom.nbond[a]] = f32(length) / dmax
    for a in range(natom):
        ia = a + 1
        molecom.xa[ia] = sysm.xa[a]
        molecom.ya[ia] = sysm.ya[a]
        molecom.za[ia] = sysm.za[a]
        molecom.itype[ia] = int(sysm.itype[a]) + 1
        molecom.qtype[ia] = 0
        molecom.mref[ia] = 0
        molecom.imageatom[ia] = 0
    for m in range(nmol):
        for a in range(int(sysm.naf[m]), int(sysm.naf[m] + sysm.nato[m])):
            molecom.mref[a + 1] = m + 1
    # grids and potential tables
    g = sysm.grid
    npt = g["npt"]
    epsr16.cellst = sysm.cellst
    epsr16.npt = npt
    epsr16.npt1 = g["npt1"]
    epsr16.npt2 = g["npt2"]
    epsr16.nptmin = g["nptmin"]
    epsr16.nptmax = g["nptmax"]
    epsr16.rejrate = f32(rejrate)
    epsr16.x[: npt + 1] = g["x"]
    epsr16.xstar[: npt + 1] = sysm.xstar
    for p in range(npairs):
        potential_par.xavs[: npt + 1, p + 1] = sysm.xavs[p]
        potential_par.xavs1[: npt + 1, p + 1] = sysm.xavs1[p]
        potential_par.ecoul[: npt + 1, p + 1] = sysm.ecoul[p]
        potential_par.ecoul1[: npt + 1, p + 1] = sysm.ecoul1[p]
    molecom.maxmolsize = f32(max(float(np.max(np.abs(np.stack([sysm.xa, sysm.ya, sysm.za])))), 0.0) * 2.0)
    for mt in range(sysm.nmoltype):
        clustercom.wholerot[mt + 1] = f32(0.0 if wholerot is None else wholerot[mt])
        clustercom.wholetrans[mt + 1] = f32(0.0 if wholetrans is None else wholetrans[mt])
    threebody_mod.nthreeb = 0
    coordconstraints_mod.ncoordconstraints = 0
    containerforces_mod.numcontainerforces = 0
    ran1com.idum = 0
    ran1com.iy = 0
    ran1com.mcall = 0
    return None


def ran1_state():
    from epsr26.common import ran1com
    return dict(idum=int(ran1com.idum), iy=int(ran1com.iy), mcall=int(ran1com.mcall),
                iv=np.array(ran1com.iv[1:33], dtype=np.int32))


def store_state():
    from epsr26.common import ergpairreference as erd
    nmol = erd.nmolhere
    return dict(nnbrefmax=int(erd.nnbrefmax), nergpair=int(erd.nergpair),
                nergpairm=np.array(erd.nergpairm[1:nmol + 1], dtype=np.int32),
                molergpair=np.array(erd.molergpair[1:, 1:nmol + 1], dtype=np.int32),
                ergpairref=np.array(erd.ergpairref[1:, 1:nmol + 1], dtype=np.int32),
                ergpair=np.array(erd.ergpair[1:erd.nergpair + 1], dtype=np.float32))


def coords_state(sysm):
    from epsr26.common import clustercom, molecom
    n, a = sysm.nmol, sysm.natom
    return dict(xa=np.array(molecom.xa[1:a + 1]), ya=np.array(molecom.ya[1:a + 1]),
                za=np.array(molecom.za[1:a + 1]),
                xadd=np.array(clustercom.xadd[1:n + 1]), yadd=np.array(clustercom.yadd[1:n + 1]),
                zadd=np.array(clustercom.zadd[1:n + 1]))


def cell_state(nmol):
    from epsr26.common import cellneighbourlist as cnl
    return dict(ncelldiva=cnl.ncelldiva, ncelldivb=cnl.ncelldivb, ncelldivc=cnl.ncelldivc, ncell=cnl.ncell,
                maxcellno=cnl.maxcellno, ncellneighb=cnl.ncellneighb,
                nmolsincell=np.array(cnl.nmolsincell[1:cnl.ncell + 1], dtype=np.int32),
                molsincell=np.array(cnl.molsincell[1:, 1:], dtype=np.int32),
                molcellno=np.array(cnl.molcellno[1:nmol + 1], dtype=np.int32),
                iacellneighb=np.array(cnl.iacellneighb[1:cnl.ncellneighb + 1], dtype=np.int32),
                ibcellneighb=np.array(cnl.ibcellneighb[1:cnl.ncellneighb + 1], dtype=np.int32),
                iccellneighb=np.array(cnl.iccellneighb[1:cnl.ncellneighb + 1], dtype=np.int32))
