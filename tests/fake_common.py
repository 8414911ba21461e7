"""Stand-ins for the reference's COMMON-block modules and routine-owning modules, filled from
a golden fixture, for the drop-in tests (the reference itself is not importable where the
GPU tests run).  Attribute names, 1-based indexing, Fortran order and the extra element 0
follow the reference's common/*.py; the values follow what tests/golden/refstate.py wrote
into the real modules when the golden was made."""

from types import SimpleNamespace as NS

import numpy as np

f32 = np.float32


def fa(*dims, dtype=f32):
    return np.zeros(tuple(int(d) + 1 for d in dims), dtype=dtype, order="F")


def common_from_golden(z):
    nmol, natom = z["sys_naf"].shape[0], z["sys_itype"].shape[0]
    ntype, npairs = int(z["sys_ntype"]), z["sys_n1extr"].shape[0]
    nmt = int(z["sys_nmoltype"])
    npt = int(z["sys_npt"])
    mpz = npt + 8
    dmax = f32(z["sys_dmax"])
    lattice = NS(cubic=True, alat=f32(1), blat=f32(1), clat=f32(1), alatx=f32(1), blaty=f32(1), clatz=f32(1),
                 blatx=f32(0), clatx=f32(0), claty=f32(0), alatc=fa(3), blatc=fa(3), clatc=fa(3))
    lattice.alatc[1] = lattice.blatc[2] = lattice.clatc[3] = f32(1)
    cc = NS(dmax=dmax, volume=f32(1), nmol=nmol, nmoltype=nmt, naf=fa(nmol, dtype=np.int32),
            nal=fa(nmol, dtype=np.int32), nato=fa(nmol, dtype=np.int32), mtype=fa(nmol, dtype=np.int32),
            ngrot=fa(nmol, dtype=np.int32), tethered=fa(nmol, dtype=bool), xadd=fa(nmol), yadd=fa(nmol),
            zadd=fa(nmol), wholerot=fa(nmt), wholetrans=fa(nmt), internrot=fa(nmt), interntrans=fa(nmt),
            nwhole=fa(2, nmt, dtype=np.int32), nmovem=fa(2, nmt, dtype=np.int32), nmovei=fa(2, nmt, dtype=np.int32),
            ninter=fa(2, nmt, dtype=np.int32), nstepreject=fa(nmol, dtype=np.int32))
    naf = z["sys_naf"].astype(np.int32) + 1
    cc.naf[1:] = naf
    cc.nato[1:] = z["sys_nato"]
    cc.nal[1:] = naf + z["sys_nato"] - 1
    cc.mtype[1:] = z["sys_mtype"] + 1
    cc.xadd[1:], cc.yadd[1:], cc.zadd[1:] = z["sys_xadd"], z["sys_yadd"], z["sys_zadd"]
    cc.wholerot[1:], cc.wholetrans[1:] = z["in_wholerot"], z["in_wholetrans"]
    mc = NS(natom=natom, natomr=int(z["in_natomr"]), ntype=ntype, npairs=npairs, dmaxmol=dmax, sizefactor=f32(1),
            simt=f32(z["sys_simt"]), stepr=f32(z["in_stepr"]), stepm=f32(z["in_stepm"]), stepri=f32(0),
            stepmi=f32(0), tolout=f32(0), tol=f32(0), tempb=f32(1), tempang=f32(1), tempangwt=f32(1),
            tempangreq=f32(1), tempdih=f32(0), tempdihwt=f32(0), tempdihreq=f32(0), cfrac=fa(ntype),
            npairref=fa(ntype, ntype, dtype=np.int32), n1extr=fa(npairs, dtype=np.int32),
            n2extr=fa(npairs, dtype=np.int32), itype=fa(natom, dtype=np.int32), xa=fa(natom), ya=fa(natom),
            za=fa(natom), maxmolsize=f32(z["in_maxmolsize"]))
    mc.cfrac[1:] = z["sys_cfrac"]
    mc.npairref[1:, 1:] = z["sys_npairref"] + 1
    mc.n1extr[1:], mc.n2extr[1:] = z["sys_n1extr"] + 1, z["sys_n2extr"] + 1
    mc.itype[1:] = z["sys_itype"] + 1
    mc.xa[1:], mc.ya[1:], mc.za[1:] = z["sys_xa"], z["sys_ya"], z["sys_za"]
    e16 = NS(cellst=f32(z["sys_cellst"]), npt=npt, npt1=int(z["sys_npt1"]), npt2=int(z["sys_npt2"]),
             nptmin=int(z["sys_nptmin"]), nptmax=int(z["sys_nptmax"]), rejrate=f32(z["in_rejrate"]), x=fa(mpz),
             xstar=fa(mpz), ycoh=fa(mpz), foqols=None, nfile=0)
    e16.x[: npt + 1] = z["sys_x"]
    e16.xstar[: npt + 1] = z["sys_xstar"]
    if "gs_foqols" in z.files:          # ycoh stays zero until the gensq stage, as when the golden was made
        e16.foqols = np.asfortranarray(z["gs_foqols"])
    pp = NS(xavs=fa(mpz, npairs), xavs1=fa(mpz, npairs), ecoul=fa(mpz, npairs), ecoul1=fa(mpz, npairs),
            irefpcof=fa(npairs, dtype=np.int32), rminex=fa(npairs), potex=fa(npairs), potexmax=fa(npairs),
            wsum=fa(4))
    for p in range(npairs):
        pp.xavs[: npt + 1, p + 1] = z["sys_xavs"][p]
        pp.xavs1[: npt + 1, p + 1] = z["sys_xavs1"][p]
        pp.ecoul[: npt + 1, p + 1] = z["sys_ecoul"][p]
        pp.ecoul1[: npt + 1, p + 1] = z["sys_ecoul1"][p]
        pp.irefpcof[p + 1] = p + 1
    pp.rminex[1:] = z["ag_rminex"] if "ag_rminex" in z.files else f32(-2.0)
    ran1com = NS(mcall=0, idum=0, iy=0, iv=fa(32, dtype=np.int32))
    cnl = NS(ncelldiva=0, ncelldivb=0, ncelldivc=0, ncelldivsq=0, ncell=0, ncellneighb=0, maxcellno=0, nmolcell=0,
             nmolsincell=None, molcellno=None, iacellneighb=None, ibcellneighb=None, iccellneighb=None,
             molsincell=None)
    erd = NS(ergpair=None, nergpair=0, nergpairmax=0, molergpair=None, ergpairref=None, nergpairm=None, nnbrefmax=0,
             ergold=None, ergnew=None, nbref=None, nnbref=0, nmolhere=0)
    mm = NS(coarsegraining=False, natomsphere=np.ones(ntype + 1, f32))
    return NS(molecom=mc, clustercom=cc, epsr16=e16, potential_par=pp, lattice=lattice, ran1com=ran1com,
              cellneighbourlist=cnl, ergpairreference=erd, molecom_mod=mm, threebody_mod=NS(nthreeb=0),
              coordconstraints_mod=NS(ncoordconstraints=0), containerforces_mod=NS(numcontainerforces=0))


def set_ran1(common, z, prefix):
    r = common.ran1com
    r.idum, r.iy, r.mcall = int(z[prefix + "idum"]), int(z[prefix + "iy"]), int(z[prefix + "mcall"])
    r.iv[1:33] = z[prefix + "iv"]


def routine_modules(z, calls):
    """Modules owning the routines; their own versions only record that they were called
    (the host fallback), except en_mole_intra, which returns the golden intra energies."""
    def rec(name, result=None):
        def f(*a):
            calls.append(name)
            return result
        return f
    eintra = z["in_eintra"]

    def en_mole_intra(im, sv, sa, sd):
        return f32(eintra[im - 1]), sv, sa, sd
    return {"cellneighbourlist": NS(initialise_cellneighbourlist=rec("host:initialise_cellneighbourlist")),
            "ato_manipulation_rev4": NS(fmolec1=rec("host:fmolec1", (0, 0, f32(0), f32(0), f32(0), f32(0))),
                                        atogen=rec("host:atogen", 0), stog=rec("host:stog"),
                                        press=rec("host:press", (f32(0), f32(0), f32(0), f32(0), f32(0))),
                                        abs_energy_ep=lambda: f32(0.0)),
            "molfit": NS(molfit=rec("host:molfit", (f32(0), f32(0), 1)), en_change=rec("host:en_change"),
                         en_mole_pair=rec("host:en_mole_pair"), en_mole_intra=en_mole_intra),
            "program": NS(gensq=rec("host:gensq"), fit_expansion=rec("host:fit_expansion"), sumgr=rec("host:sumgr"),
                          sumsq=rec("host:sumsq"), generate_ep=rec("host:generate_ep"),
                          generate_rp=rec("host:generate_rp"))}


class GroupsGolden:
    """A rotational-group golden (rot.npz and its kind) seen under the key names the COMMON
    stand-ins read."""
    ALIAS = {"in_wholerot": "wholerot_in", "in_wholetrans": "wholetrans_in", "in_eintra": "eintra"}

    def __init__(self, z):
        self.z = z

    def __getitem__(self, k):
        return self.z[self.ALIAS.get(k, k)]

    @property
    def files(self):
        return list(self.z.files) + list(self.ALIAS)


def common_with_groups(name, shake=False):
    """COMMON stand-ins and routine modules for a rotational-group golden (tests/golden/rot.npz,
    shake_rot.npz, dih_rot.npz, dih_shake.npz): the intramolecular model, the groups 1-based as
    the reference holds them (molecom_mod labaxi/rotf/rotl/labrot, clustercom ngrot/nrf/nrl) and,
    for the DIH goldens, the dihedral angles (molecom labrotdih/ndihedralang/dihedralang,
    tempdihreq 1).  Returns (golden, common, modules, calls)."""
    from tests.goldens import GOLDEN
    z = np.load(GOLDEN + "/" + name)
    p = GroupsGolden(z)
    calls = []
    mods = routine_modules(p, calls)
    c = common_from_golden(p)
    mc, cc, pp = c.molecom, c.clustercom, c.potential_par
    natom, nmol, ntype = mc.natom, cc.nmol, mc.ntype
    npairs, npt = mc.npairs, c.epsr16.npt
    iab = z["iabond"]
    mb = iab.shape[1]
    mc.nbond = fa(natom, dtype=np.int32)
    mc.nbond[1:] = z["nbond"]
    mc.iabond = fa(natom, mb, dtype=np.int32)
    mc.iabond[1:, 1:] = iab + 1
    mc.tbond = fa(natom, mb)
    mc.tbond[1:, 1:] = z["tbond"]
    mc.imageatom, mc.qtype = fa(natom, dtype=np.int32), fa(natom, dtype=np.int32)
    mc.amassa, mc.amassr = fa(ntype), fa(npairs)
    mc.amassa[1:], mc.amassr[1:] = z["amassa"], z["amassr"]
    sc = z["scal"]
    mc.sizefactor, mc.tempb, mc.tempangreq, mc.tempangwt = f32(sc[1]), f32(sc[2]), f32(sc[3]), f32(sc[3])
    mc.refine_intra, mc.refine_intra_fac, mc.stepri = False, f32(0.0), f32(1.0)
    mpz = pp.xavs.shape[0] - 1
    pp.xav, pp.xav1 = fa(mpz, npairs), fa(mpz, npairs)
    pp.xav[: npt + 1, 1:], pp.xav1[: npt + 1, 1:] = z["xav"].T, z["xav1"].T
    cc.internrot[1:] = z["internrot_in"]
    if shake:
        mc.stepmi = f32(z["stepmi"])
        cc.interntrans[1:] = z["interntrans_in"]
    # the rotational groups, 1-based as the reference holds them
    ng = z["rot_first"].size
    cc.ngrot[1:] = z["ngrot"]
    cc.nrf, cc.nrl = fa(nmol, dtype=np.int32), fa(nmol, dtype=np.int32)
    cc.nrf[1:], cc.nrl[1:] = z["rot_nrf"] + 1, z["rot_nrl"] + 1
    lab = fa(ng, 2, dtype=np.int32)
    lab[1:, 1:] = z["rot_axis"] + 1
    rotf, rotl = fa(ng, dtype=np.int32), fa(ng, dtype=np.int32)
    rotf[1:], rotl[1:] = z["rot_first"] + 1, z["rot_last"] + 1
    labrot = fa(z["rot_atoms"].size, dtype=np.int32)
    labrot[1:] = z["rot_atoms"] + 1
    dih = "dih_cos" in z.files
    c.molecom_mod = NS(coarsegraining=False, natomsphere=c.molecom_mod.natomsphere, ngrrot=ng,
                       rotgrp=np.array(["   "] + ["DIH" if dih else "ROT"] * ng, dtype=object), labaxi=lab,
                       rotf=rotf, rotl=rotl, labrot=labrot, nrottot=int(z["rot_atoms"].size))
    mc.ndihedralang = fa(ng, dtype=np.int32)
    if dih:
        # one dihedral angle per group, as the reference held them (1.0 and 2.5 rad alternately)
        mc.ndihedralang[1:] = np.diff(z["dih_grp0"])
        mc.labrotdih = np.zeros((3, 2, ng + 1), np.int32)
        mc.dihedralang = np.zeros((2, ng + 1), f32)
        for ir in range(1, ng + 1):
            mc.labrotdih[1, 1, ir], mc.labrotdih[2, 1, ir] = z["dih_atoms"][ir - 1] + 1
            mc.dihedralang[1, ir] = f32(1.0) if (ir - 1) % 2 == 0 else f32(2.5)
        mc.tempdihreq = mc.tempdihwt = f32(1.0)
        mc.tempdih = f32(f32(mc.tempdihwt) * f32(mc.tempb))
    return z, c, mods, calls
