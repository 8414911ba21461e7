"""Drop-in replacements for the reference's pair-path routines, with their signatures.

The reference translation (package ``epsr26``) keeps its state in COMMON-block modules
(``epsr26.common.molecom``, ``clustercom``, ``epsr16``, ``potential_par``, ``lattice``,
``ran1com``, ``cellneighbourlist``, ``ergpairreference``, ``molecom_mod`` ...) as 1-based,
Fortran-ordered NumPy arrays, and its callers look routines up through their module at
call time.  ``PairPath`` holds a ``DeviceBox`` mirror of that state and provides, with the
reference's argument lists and return values:

* ``initialise_cellneighbourlist`` (library/cellneighbourlist.py:23)
* ``fmolec1`` (library/ato_manipulation_rev4.py:2374)
* ``molfit`` (library/molfit.py:52), whole-molecule branch
* ``en_change`` / ``en_mole_pair`` (library/molfit.py:806 / :1528)
* ``atogen`` (library/ato_manipulation_rev4.py:3640)
* ``gensq`` (programs/epsr_standalone_rev3.py:4731)
* ``stog`` (library/ato_manipulation_rev4.py:4067)
* ``fit_expansion`` (programs/epsr_standalone_rev3.py:4806)
* ``press`` (library/ato_manipulation_rev4.py:3903)
* ``sumgr`` / ``sumsq`` (programs/epsr_standalone_rev3.py:3578 / :3642)
* ``generate_ep`` (programs/epsr_standalone_rev3.py:5876)
* ``generate_rp`` (programs/epsr_standalone_rev3.py:5675, with generate_mp)

``install()`` assigns them onto the given modules (the reference's own rerouting
mechanism, trace.py:94-125) and keeps the originals.

State protocol.  Every call is synchronous, as the reference's routines are.  On entry
the wrapper compares the COMMON arrays it depends on with what it last wrote or uploaded
(coordinates, potential tables, stored pair energies) and uploads what the host changed;
the ran1 state is always uploaded.  On return it writes everything the routine changes
back into the COMMON arrays in place (same array objects, so aliases held by other
routines stay valid).  A call that needs a feature outside the pair path (rotational
groups of a type other than ROT or DIH, tethering, three-body terms,
coordination constraints, container forces, coarse graining, molecules of more than 64 atoms)
runs the reference's own routine on the host instead; the next device call picks up whatever
it changed.

The cell list must come from the installed ``initialise_cellneighbourlist`` (the
reference loop rebuilds it every iteration, epsr_standalone_rev3.py:1265); a cell list
built elsewhere is detected and refused with ``EpsrGpuError``.  Log lines the reference
writes to unit 6 inside these routines are not reproduced.
"""

from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib, transforms
from ._lib import EpsrGpuError, check
from .box import BoxArrays, Ran1State, trsteps

f32 = np.float32
ROUTINES = ("initialise_cellneighbourlist", "fmolec1", "molfit", "atogen", "stog", "gensq", "fit_expansion",
            "press", "sumgr", "sumsq", "generate_ep", "generate_rp", "en_change", "en_mole_pair")
# en_change / en_mole_pair are per-molecule calls: rerouting them makes every host caller
# (including host fallbacks) launch one kernel per call, so they are installed only on request.
DEFAULT_ROUTINES = tuple(r for r in ROUTINES if r not in ("en_change", "en_mole_pair"))
# module that owns each routine in the reference
OWNER = {"initialise_cellneighbourlist": "cellneighbourlist", "fmolec1": "ato_manipulation_rev4",
         "atogen": "ato_manipulation_rev4", "stog": "ato_manipulation_rev4", "press": "ato_manipulation_rev4",
         "molfit": "molfit",
         "en_change": "molfit", "en_mole_pair": "molfit", "gensq": "program", "fit_expansion": "program",
         "sumgr": "program", "sumsq": "program", "generate_ep": "program", "generate_rp": "program"}


def _fortran(shape, dtype):
    """A zeroed 1-based Fortran-order array of the reference's form (extent + 1 per axis)."""
    return np.zeros(tuple(int(s) + 1 for s in shape), dtype=dtype, order="F")


def _mcall_advance(old, dev32):
    """The reference's ran1 call counter (a Python int) after the device advanced its
    32-bit copy from ``old`` to ``dev32``."""
    return int(old) + ((int(np.int64(dev32) & 0xFFFFFFFF) - (int(old) & 0xFFFFFFFF)) & 0xFFFFFFFF)


def _idiv(a, b):
    """Fortran integer division (truncation toward zero)."""
    q = abs(int(a)) // abs(int(b))
    return q if (a >= 0) == (b > 0) else -q


class PairPath:
    """The GPU pair path bound to one set of COMMON-block modules.

    ``common``: an object whose attributes are the reference's COMMON modules (the
    package ``epsr26.common`` itself).  ``modules``: the modules that own the routines,
    keyed ``cellneighbourlist`` (library), ``ato_manipulation_rev4``, ``molfit`` and
    ``program`` (the loaded ``epsr`` program module holding gensq and fit_expansion).
    ``strict``: 1 runs the sequential MC kernel and the reference's float32 summation
    order everywhere (bit-identical apart from transcendentals); 0 runs the speculative
    MC cycle and double sums (within the stated tolerance).
    """

    def __init__(self, common, modules, strict=False, device="cuda"):
        self.c = common
        self.mods = dict(modules)
        self.strict = bool(strict)
        self.device = device
        self.orig = {}
        self.d = None
        self._snap = {}
        self._mirror_ok = False
        self.cos_override = None      # test hook: [3*nmol] cosines for the next molfit call

    # ------------------------------------------------------------------ install
    def install(self, routines=DEFAULT_ROUTINES):
        for name in routines:
            mod = self.mods[OWNER[name]]
            if name not in self.orig:
                self.orig[name] = getattr(mod, name)
            setattr(mod, name, getattr(self, name))
        return self

    def uninstall(self):
        for name, f in self.orig.items():
            setattr(self.mods[OWNER[name]], name, f)
        self.orig = {}

    def _host(self, name, *args):
        """Run the reference's own routine (the one replaced at install, else the module's)."""
        f = self.orig.get(name) or getattr(self.mods[OWNER[name]], name)
        return f(*args)

    # ------------------------------------------------------------------ COMMON -> host box
    def box_from_common(self) -> BoxArrays:
        c = self.c
        mc, cc, e16, pp, lat = c.molecom, c.clustercom, c.epsr16, c.potential_par, c.lattice
        nmol, natom, ntype, npairs = int(cc.nmol), int(mc.natom), int(mc.ntype), int(mc.npairs)
        npt = int(e16.npt)
        ld = npt + 1
        tab = lambda a: np.ascontiguousarray(np.asarray(a)[:ld, 1:npairs + 1].T, dtype=f32)  # noqa: E731
        return BoxArrays(
            naf=np.asarray(cc.naf[1:nmol + 1], np.int32) - 1, nato=np.asarray(cc.nato[1:nmol + 1], np.int32),
            mtype=np.asarray(cc.mtype[1:nmol + 1], np.int32) - 1,
            itype=np.asarray(mc.itype[1:natom + 1], np.int32) - 1,
            xa=np.array(mc.xa[1:natom + 1], f32), ya=np.array(mc.ya[1:natom + 1], f32),
            za=np.array(mc.za[1:natom + 1], f32), xadd=np.array(cc.xadd[1:nmol + 1], f32),
            yadd=np.array(cc.yadd[1:nmol + 1], f32), zadd=np.array(cc.zadd[1:nmol + 1], f32),
            npairref=np.ascontiguousarray(np.asarray(mc.npairref)[1:ntype + 1, 1:ntype + 1], np.int32) - 1,
            n1extr=np.asarray(mc.n1extr[1:npairs + 1], np.int32) - 1,
            n2extr=np.asarray(mc.n2extr[1:npairs + 1], np.int32) - 1,
            nmoltype=int(cc.nmoltype), dmax=f32(cc.dmax), cellst=f32(e16.cellst),
            x=np.array(e16.x[:ld], f32), xstar=np.array(e16.xstar[:ld], f32), npt=npt, npt1=int(e16.npt1),
            npt2=int(e16.npt2), nptmax=int(e16.nptmax), xavs=tab(pp.xavs), xavs1=tab(pp.xavs1),
            ecoul=tab(pp.ecoul), ecoul1=tab(pp.ecoul1), simt=f32(mc.simt),
            cfrac=np.array(mc.cfrac[1:ntype + 1], f32), natomr=int(mc.natomr), cubic=bool(lat.cubic),
            lat6=np.array([lat.alatx, lat.blatx, lat.clatx, lat.blaty, lat.claty, lat.clatz], f32),
            lat9=np.array(list(lat.alatc[1:4]) + list(lat.blatc[1:4]) + list(lat.clatc[1:4]), f32),
            maxmolsize=f32(mc.maxmolsize))

    # ------------------------------------------------------------------ state sync
    @staticmethod
    def _topology(b):
        return (b.nmol, b.natom, b.ntype, b.npairs, b.nmoltype, b.npt, b.npt1, b.npt2, b.cubic,
                b.naf.tobytes(), b.nato.tobytes(), b.mtype.tobytes(), b.itype.tobytes(), b.npairref.tobytes(),
                b.n1extr.tobytes(), b.n2extr.tobytes(), b.lat6.tobytes(), float(b.dmax), float(b.cellst))

    @staticmethod
    def _tables(b):
        return (b.xavs, b.xavs1, b.ecoul, b.ecoul1, b.xstar, b.cfrac)

    def _sync_in(self):
        """Bring the device mirror up to date with the COMMON blocks; returns the host box."""
        from .device import DeviceBox
        b = self.box_from_common()
        topo = self._topology(b)
        s = self._snap
        if self.d is None or s.get("topo") != topo:
            self.d = DeviceBox(b, device=self.device)
            self._mirror_ok = False
            s.clear()
            s["topo"] = topo
        elif any(not np.array_equal(u, v) for u, v in zip(self._tables(b), s["tables"])) \
                or float(b.simt) != s["simt"] or int(b.natomr) != s["natomr"]:
            self.d.upload(b)                   # tables changed (generate_ep): full re-upload
        elif any(not np.array_equal(getattr(b, k), s["coords"][k]) for k in ("xa", "ya", "za", "xadd", "yadd",
                                                                              "zadd")):
            self.d.host = b
            self.d.upload_coords(b.xa, b.ya, b.za, b.xadd, b.yadd, b.zadd)
        else:
            self.d.host = b
        s["tables"] = tuple(np.array(t) for t in self._tables(b))
        s["simt"], s["natomr"] = float(b.simt), int(b.natomr)
        s["coords"] = {k: np.array(getattr(b, k)) for k in ("xa", "ya", "za", "xadd", "yadd", "zadd")}
        return b

    def _coords_out(self):
        co = self.d.download_coords()
        mc, cc = self.c.molecom, self.c.clustercom
        na, nm = co["xa"].shape[0], co["xadd"].shape[0]
        mc.xa[1:na + 1], mc.ya[1:na + 1], mc.za[1:na + 1] = co["xa"], co["ya"], co["za"]
        cc.xadd[1:nm + 1], cc.yadd[1:nm + 1], cc.zadd[1:nm + 1] = co["xadd"], co["yadd"], co["zadd"]
        self._snap["coords"] = {k: np.array(v) for k, v in co.items()}

    def _ran1_in(self):
        r = self.c.ran1com
        st = Ran1State(idum=int(r.idum), iy=int(r.iy), mcall=int(np.int64(r.mcall) & 0xFFFFFFFF),
                       iv=np.asarray(r.iv[1:33], np.int32).copy())
        self._mcall0 = int(r.mcall)
        return self.d.ran1_tensor(st)

    def _ran1_out(self, t):
        torch.cuda.synchronize()
        a = t.cpu().numpy()
        r = self.c.ran1com
        r.idum, r.iy = int(a[0]), int(a[1])
        r.iv[1:33] = a[3:35]
        r.mcall = _mcall_advance(self._mcall0, a[2])

    def _check_cells(self):
        cnl = self.c.cellneighbourlist
        s = self._snap.get("cells")
        if self.d.cells is None or s is None or cnl.molcellno is None or \
                not np.array_equal(np.asarray(cnl.molcellno[1:]), s["molcellno"]) or \
                not np.array_equal(np.asarray(cnl.nmolsincell[1:]), s["nmolsincell"]) or \
                int(cnl.ncellneighb) != s["ncellneighb"]:
            raise EpsrGpuError(4, "cell list was not built by the GPU initialise_cellneighbourlist")

    def _store_in(self):
        """Upload pair energies (or the whole store) that the host changed since the last sync."""
        erd = self.c.ergpairreference
        s = self._snap.get("store")
        if s is None:
            raise EpsrGpuError(4, "pair store was not built by the GPU fmolec1")
        nmol, M = self.d.host.nmol, int(erd.nnbrefmax)
        n = int(erd.nergpair)
        nm = np.asarray(erd.nergpairm[1:nmol + 1], np.int32)
        mol = np.ascontiguousarray(np.asarray(erd.molergpair)[1:M + 1, 1:nmol + 1].T, np.int32) - 1
        ref = np.ascontiguousarray(np.asarray(erd.ergpairref)[1:M + 1, 1:nmol + 1].T, np.int32)
        erg = np.array(erd.ergpair[1:n + 1], f32)
        if M != s["M"] or n != s["n"] or not (np.array_equal(nm, s["nergpairm"]) and np.array_equal(mol, s["mol"])
                                             and np.array_equal(ref, s["ref"])):
            if M != self.d.nnbrefmax or n > self.d.s_erg.numel():
                raise EpsrGpuError(4, "pair store resized outside the GPU path")
            d = self.d
            d.s_nergpairm[:nmol].copy_(torch.from_numpy(nm))
            d.s_mol[:nmol * M].copy_(torch.from_numpy(mol.reshape(-1)))
            d.s_ref[:nmol * M].copy_(torch.from_numpy(ref.reshape(-1)))
            d.s_n[:1].copy_(torch.tensor([n], dtype=torch.int32))
            self._mirror_ok = False            # the fast sweep's mirror index is stale
        if not np.array_equal(erg, s["erg"]):
            self.d.s_erg[:n].copy_(torch.from_numpy(erg))
        s.update(M=M, n=n, nergpairm=nm, mol=mol, ref=ref, erg=erg)

    def _store_out(self, values_only):
        erd = self.c.ergpairreference
        st = self.d.download_store()
        nmol, M, n = self.d.host.nmol, st["nnbrefmax"], st["nergpair"]
        if not values_only:
            # allocation of initialise_ergpair (ergpairreference.py:63-100) and the 20%
            # growth of reallocate_ergpair (:128-147) for n stored energies
            cap = 100 * nmol
            while n > cap:
                cap = _idiv((cap + 10) * 12, 10)
            erd.nmolhere = nmol
            erd.nnbrefmax = M
            erd.nergpairmax = cap
            erd.ergpair = _fortran((cap,), f32)
            erd.molergpair = _fortran((M, nmol), np.int32)
            erd.ergpairref = _fortran((M, nmol), np.int32)
            erd.nergpairm = _fortran((nmol,), np.int32)
            erd.nnbref = 0
            erd.ergold = _fortran((M,), f32)
            erd.ergnew = _fortran((M,), f32)
            erd.nbref = _fortran((M,), np.int32)
            mol = st["molergpair"].copy()
            for im in range(nmol):                 # unused slots stay 0 as in the reference
                mol[im, st["nergpairm"][im]:] = -1
            erd.molergpair[1:M + 1, 1:nmol + 1] = (mol + 1).T
            ref = st["ergpairref"].copy()
            for im in range(nmol):
                ref[im, st["nergpairm"][im]:] = 0
            erd.ergpairref[1:M + 1, 1:nmol + 1] = ref.T
            erd.nergpairm[1:nmol + 1] = st["nergpairm"]
            erd.nergpair = n
        erd.ergpair[1:n + 1] = st["ergpair"]
        nm = np.asarray(erd.nergpairm[1:nmol + 1], np.int32)
        self._snap["store"] = dict(
            M=M, n=n, nergpairm=nm,
            mol=np.ascontiguousarray(np.asarray(erd.molergpair)[1:M + 1, 1:nmol + 1].T, np.int32) - 1,
            ref=np.ascontiguousarray(np.asarray(erd.ergpairref)[1:M + 1, 1:nmol + 1].T, np.int32),
            erg=np.array(st["ergpair"], f32))

    # ------------------------------------------------------------------ feature checks
    def _outside_path(self):
        c = self.c
        nmol = int(c.clustercom.nmol)
        if getattr(c.molecom_mod, "coarsegraining", False):
            return True
        if int(getattr(c.threebody_mod, "nthreeb", 0)) > 0:
            return True
        if int(getattr(c.coordconstraints_mod, "ncoordconstraints", 0)) > 0:
            return True
        if float(getattr(c.containerforces_mod, "numcontainerforces", 0)) > 0.0:
            return True
        teth = getattr(c.clustercom, "tethered", None)
        if teth is not None and bool(np.any(np.asarray(teth[1:nmol + 1]))):
            return True
        return int(np.max(np.asarray(c.clustercom.nato[1:nmol + 1]))) > 64

    # ------------------------------------------------------------------ routines
    def initialise_cellneighbourlist(self, nmolcellin, xadd, yadd, zadd, nmol, rmax):
        """cellneighbourlist.py:23-90: fills the COMMON cell arrays (molsincell, offsets...)."""
        cnl = self.c.cellneighbourlist
        cnl.nmolcell = min(int(nmolcellin), int(nmol))
        cc = self.c.clustercom
        if xadd is not cc.xadd or yadd is not cc.yadd or zadd is not cc.zadd or int(nmol) != int(cc.nmol):
            return self._host("initialise_cellneighbourlist", nmolcellin, xadd, yadd, zadd, nmol, rmax)
        self._sync_in()
        self.d.cell_list(int(nmolcellin), f32(rmax))
        cl = self.d.download_cells()
        ncell, mx = int(cl["ncell"]), int(cl["maxcellno"])
        cnl.ncelldiva, cnl.ncelldivb, cnl.ncelldivc = int(cl["ncelldiva"]), int(cl["ncelldivb"]), int(cl["ncelldivc"])
        cnl.ncell = ncell
        cnl.ncelldivsq = cnl.ncelldiva * cnl.ncelldivb
        cnl.maxcellno = mx
        cnl.ncellneighb = int(cl["ncellneighb"])
        start, mols = cl["cell_start"], cl["cell_mols"]
        counts = np.diff(start[:ncell + 1]).astype(np.int32)
        cnl.nmolsincell = _fortran((ncell,), np.int32)
        cnl.nmolsincell[1:] = counts
        cnl.molcellno = _fortran((int(nmol),), np.int32)
        cnl.molcellno[1:] = cl["molcellno"][: int(nmol)]
        cnl.molsincell = _fortran((mx, ncell), np.int32)
        for c in range(ncell):
            k = int(counts[c])
            if k:
                cnl.molsincell[1:k + 1, c + 1] = mols[start[c]:start[c] + k] + 1
        for i, name in enumerate(("iacellneighb", "ibcellneighb", "iccellneighb")):
            a = _fortran((ncell,), np.int32)
            a[1:cnl.ncellneighb + 1] = cl["offsets"][:, i]
            setattr(cnl, name, a)
        self._snap["cells"] = dict(molcellno=np.array(cnl.molcellno[1:]), nmolsincell=np.array(cnl.nmolsincell[1:]),
                                   ncellneighb=int(cnl.ncellneighb))
        return None

    def fmolec1(self, ierr, num_threads_input, ftest, ftestb, ftethered, fcoordconstraints):
        """ato_manipulation_rev4.py:2374-2528: rebuilds the pair store in the COMMON block;
        returns (ierr, num_threads_input, ftest, ftestb, ftethered, fcoordconstraints)."""
        if self._outside_path():
            return self._host("fmolec1", ierr, num_threads_input, ftest, ftestb, ftethered, fcoordconstraints)
        if num_threads_input <= 0:
            num_threads_input = 0          # idiv(omp_get_max_threads(), 2) with the reference's 1-thread stubs
        mc = self.c.molecom
        mc.tempangwt = mc.tempangreq
        mc.tempdihwt = mc.tempdihreq
        mc.tempang = mc.tempangwt
        mc.tempdih = f32(f32(mc.tempdihwt) * f32(mc.tempb))
        b = self._sync_in()
        self._check_cells()
        model = self._intra_model(b, allow_rot=self._rot_groups() is not None)
        if model is not None:
            # intramolecular energies (molfit.py:1327) on the device
            eintra = model.en_mole_intra()
        else:
            # rotational groups of another type: the reference's own host routine
            en_mole_intra = self.mods["molfit"].en_mole_intra
            sv = sa = sd = f32(0.0)
            eintra = np.zeros(b.nmol, f32)
            for im in range(1, b.nmol + 1):
                e, sv, sa, sd = en_mole_intra(im, sv, sa, sd)
                eintra[im - 1] = e
        ft, fb = self.d.fmolec1(eintra, strict=True)
        self._store_out(values_only=False)
        self._mirror_ok = True
        nmol = f32(b.nmol)
        return 0, num_threads_input, f32(ft), f32(fb), f32(0.0) / nmol, f32(0.0) / nmol

    def _rot_groups(self):
        """The box's rotational groups as the device takes them -- (nrf, nrl, axis, first, last,
        atoms), 0-based -- when every group is of type ROT or DIH; () when no molecule has
        groups; None otherwise (the host runs what needs them)."""
        c = self.c
        cc = c.clustercom
        nmol = int(cc.nmol)
        ngrot = np.asarray(cc.ngrot[1:nmol + 1])
        if not bool(np.any(ngrot > 0)):
            return ()
        mm = getattr(c, "molecom_mod", None)
        if mm is None or getattr(mm, "labaxi", None) is None:
            return None
        ng = int(mm.ngrrot)
        if any(str(mm.rotgrp[i]).strip() not in ("ROT", "DIH") for i in range(1, ng + 1)):
            return None
        if self._dihedrals(ng) is False:
            return None
        nrot = int(mm.nrottot)
        return (np.asarray(cc.nrf[1:nmol + 1], np.int32) - 1, np.asarray(cc.nrl[1:nmol + 1], np.int32) - 1,
                np.asarray(mm.labaxi)[1:ng + 1, 1:3].astype(np.int32) - 1,
                np.asarray(mm.rotf[1:ng + 1], np.int32) - 1, np.asarray(mm.rotl[1:ng + 1], np.int32) - 1,
                np.asarray(mm.labrot[1:nrot + 1], np.int32) - 1)

    def _dihedrals(self, ng=None):
        """The rotational groups' dihedral angles as the device's intramolecular model takes
        them (molecom labrotdih / ndihedralang / dihedralang, molecom_mod rotgrp): a dict, or
        None when no group has any; False when a group has dihedral angles but the COMMON blocks
        do not carry their atoms or angles."""
        from .box import libm_f1
        c = self.c
        cc, mc = c.clustercom, c.molecom
        mm = getattr(c, "molecom_mod", None)
        if mm is None or getattr(mm, "labaxi", None) is None:
            return None
        ng = int(mm.ngrrot) if ng is None else ng
        nd = getattr(mc, "ndihedralang", None)
        isdih = np.array([1 if str(mm.rotgrp[i]).strip() == "DIH" else 0 for i in range(1, ng + 1)], np.int32)
        ndih = np.zeros(ng, np.int32) if nd is None else np.asarray(nd[1:ng + 1], np.int32)
        if not bool(np.any(ndih > 0)) and not bool(np.any(isdih)):
            return None
        if bool(np.any(ndih > 0)) and (getattr(mc, "labrotdih", None) is None or getattr(mc, "dihedralang", None) is None):
            return False
        nmol = int(cc.nmol)
        atoms, cs, sn = [], [], []
        for ir in range(1, ng + 1):
            for kd in range(1, int(ndih[ir - 1]) + 1):
                atoms.append((int(mc.labrotdih[1, kd, ir]) - 1, int(mc.labrotdih[2, kd, ir]) - 1))
                a = f32(mc.dihedralang[kd, ir])
                cs.append(libm_f1("cosf", a))
                sn.append(libm_f1("sinf", a))
        return dict(grp_nrf=np.asarray(cc.nrf[1:nmol + 1], np.int32) - 1, grp_nrl=np.asarray(cc.nrl[1:nmol + 1], np.int32) - 1,
                    grp_axis=np.asarray(mm.labaxi)[1:ng + 1, 1:3].astype(np.int32) - 1,
                    grp_dih0=np.concatenate([[0], np.cumsum(ndih)]).astype(np.int32), grp_isdih=isdih,
                    dih_atoms=np.array(atoms, np.int32).reshape(-1, 2), dih_cos=np.array(cs, f32),
                    dih_sin=np.array(sn, f32), tempdih=f32(mc.tempdih))

    def _intra_model(self, b, allow_rot=False):
        """The device intramolecular model (en_atom_intra molfit.py:923) from molecom, or None
        when the COMMON blocks carry no bond lists, or when a molecule has rotational groups and
        allow_rot is false; with allow_rot the groups' dihedral angles come with it."""
        from .intra import IntraModel
        c = self.c
        mc, cc, pp, e16 = c.molecom, c.clustercom, c.potential_par, c.epsr16
        nmol, natom, npairs = b.nmol, b.natom, b.npairs
        ngrot = np.asarray(cc.ngrot[1:nmol + 1], np.int32)
        if getattr(mc, "nbond", None) is None or getattr(pp, "xav", None) is None or \
                (bool(np.any(ngrot > 0)) and not allow_rot):
            return None
        nb = np.asarray(mc.nbond[1:natom + 1], np.int32)
        mb = max(1, int(nb.max()) if natom else 1)
        ld = b.npt + 1
        return IntraModel(self.d, nbond=nb, iabond=np.asarray(mc.iabond)[1:natom + 1, 1:mb + 1].astype(np.int32) - 1,
                          tbond=np.asarray(mc.tbond)[1:natom + 1, 1:mb + 1].astype(f32),
                          imageatom=np.asarray(mc.imageatom[1:natom + 1], np.int32) - 1,
                          qtype=np.asarray(mc.qtype[1:natom + 1], np.int32),
                          amassa=np.asarray(mc.amassa[1:b.ntype + 1], f32), amassr=np.asarray(mc.amassr[1:npairs + 1], f32),
                          xav=np.asarray(pp.xav)[:ld, 1:npairs + 1].T, xav1=np.asarray(pp.xav1)[:ld, 1:npairs + 1].T,
                          stepcl=f32(e16.cellst) / f32(mc.dmaxmol), simt=f32(mc.simt), sizefactor=f32(mc.sizefactor),
                          tempb=f32(mc.tempb), tempang=f32(mc.tempang), refine_intra=bool(getattr(mc, "refine_intra", False)),
                          refine_intra_fac=f32(getattr(mc, "refine_intra_fac", 0.0)), ngrot=ngrot,
                          dih=self._dihedrals() if allow_rot and bool(np.any(ngrot > 0)) else None)

    def molfit(self, fadds, faddbs, nisum, intra, rotfreq, ireset):
        """molfit.py:52-541: the whole-molecule branch and the intramolecular branch (:124-267),
        internal rotations of ROT and DIH groups included, on the device; returns (fadds, faddbs, nisum)."""
        c = self.c
        mc, cc = c.molecom, c.clustercom
        nmol = int(cc.nmol)
        groups = self._rot_groups()
        rotcycle = nisum == rotfreq * _idiv(nisum, rotfreq)
        if nisum >= intra and not self._outside_path():
            r = self._molfit_intra(fadds, faddbs, ireset)
            if r is not None:
                return r
        if nisum >= intra or groups is None or self._outside_path():
            return self._host("molfit", fadds, faddbs, nisum, intra, rotfreq, ireset)
        b = self._sync_in()
        self._check_cells()
        self._store_in()
        # host-side prologue of molfit (:87-118)
        mc.tol = f32(mc.tolout) / f32(cc.dmax)
        nmt = int(cc.nmoltype)
        for name in ("nmovei", "ninter", "nwhole", "nmovem"):
            getattr(cc, name)[1:3, 1:nmt + 1] = 0
        mc.tempang = mc.tempangwt
        mc.tempdih = f32(f32(mc.tempdihwt) * f32(mc.tempb))
        tmax, tmin = trsteps(b.natomr)
        d = self.d
        d.mc_setup(rejrate=f32(c.epsr16.rejrate), stepr=f32(mc.stepr), stepm=f32(mc.stepm),
                   wholerot=np.asarray(cc.wholerot[1:nmt + 1], f32), wholetrans=np.asarray(cc.wholetrans[1:nmt + 1], f32),
                   internrot=np.asarray(cc.internrot[1:nmt + 1], f32),
                   interntrans=np.asarray(cc.interntrans[1:nmt + 1], f32),
                   nstepreject=np.asarray(cc.nstepreject[1:nmol + 1], np.int32), ran1=Ran1State(),
                   trstepmax=tmax, trstepmin=tmin, ireset=int(ireset), fadds=f32(fadds))
        d.m_ran1 = self._ran1_in()
        d.cmc.ran1 = C.c_void_p(d.m_ran1.data_ptr())
        if groups:
            # internal rotations of the ROT groups every rotfreq cycles (molfit.py:295-360)
            d.set_rotations(self._intra_model(b, allow_rot=True), *groups, stepri=f32(mc.stepri), faddbs=f32(faddbs))
        cos = self.cos_override
        self.cos_override = None
        d.molfit(strict=self.strict or not self._mirror_ok, cos_override=cos, rotcycle=rotcycle)
        d.check_status()
        out = d.download_mc()
        self._ran1_out(d.m_ran1)
        cc.wholerot[1:nmt + 1], cc.wholetrans[1:nmt + 1] = out["wholerot"], out["wholetrans"]
        cc.internrot[1:nmt + 1], cc.interntrans[1:nmt + 1] = out["internrot"], out["interntrans"]
        cc.nwhole[1:3, 1:nmt + 1] = out["nwhole"]
        cc.nmovem[1:3, 1:nmt + 1] = out["nmovem"]
        cc.nstepreject[1:nmol + 1] = out["nstepreject"]
        self._coords_out()
        self._store_out(values_only=True)
        if groups:
            cc.ninter[1:3, 1:nmt + 1] = d.m_ninter.cpu().numpy().reshape(2, nmt)
            faddbs = f32(d.m_faddbs.cpu().numpy()[0])
        else:
            faddbs = f32(faddbs) + f32(0.0) / f32(nmol)     # faddb stays 0 without internal rotations
        return out["fadds"], faddbs, nisum + 1

    def _molfit_intra(self, fadds, faddbs, ireset):
        """The intramolecular cycle of molfit (:119-267, step adaptation :465-536) on the
        device, the internal rotations of ROT and DIH groups included; None when a group is of
        another type, or the COMMON blocks carry no bond lists (the host runs the cycle)."""
        c = self.c
        mc, cc = c.molecom, c.clustercom
        nmol = int(cc.nmol)
        groups = self._rot_groups()
        if groups is None or getattr(mc, "nbond", None) is None:
            return None
        b = self._sync_in()
        self._check_cells()
        self._store_in()
        mc.tol = f32(mc.tolout) / f32(cc.dmax)
        nmt = int(cc.nmoltype)
        for name in ("nmovei", "ninter", "nwhole", "nmovem"):
            getattr(cc, name)[1:3, 1:nmt + 1] = 0
        mc.tempang = mc.tempangwt
        mc.tempdih = f32(f32(mc.tempdihwt) * f32(mc.tempb))
        model = self._intra_model(b, allow_rot=bool(groups))
        tmax, tmin = trsteps(b.natomr)
        d = self.d
        d.mc_setup(rejrate=f32(c.epsr16.rejrate), stepr=f32(mc.stepr), stepm=f32(mc.stepm),
                   wholerot=np.asarray(cc.wholerot[1:nmt + 1], f32), wholetrans=np.asarray(cc.wholetrans[1:nmt + 1], f32),
                   internrot=np.asarray(cc.internrot[1:nmt + 1], f32),
                   interntrans=np.asarray(cc.interntrans[1:nmt + 1], f32),
                   nstepreject=np.asarray(cc.nstepreject[1:nmol + 1], np.int32), ran1=Ran1State(),
                   trstepmax=tmax, trstepmin=tmin, ireset=int(ireset), fadds=f32(fadds))
        d.m_ran1 = self._ran1_in()
        d.cmc.ran1 = C.c_void_p(d.m_ran1.data_ptr())
        if groups:
            # each molecule's groups rotated after its atom moves (:175-245)
            d.set_rotations(model, *groups, stepri=f32(mc.stepri), faddbs=f32(faddbs))
        cos = self.cos_override
        self.cos_override = None
        d.set_cos_override(cos)
        fb = torch.tensor([float(f32(faddbs))], dtype=torch.float32, device=d.dev)
        nmovei = model.molfit_shake(f32(mc.stepmi), fb).cpu().numpy()
        d.check_status()
        out = d.download_mc()
        self._ran1_out(d.m_ran1)
        cc.wholerot[1:nmt + 1], cc.wholetrans[1:nmt + 1] = out["wholerot"], out["wholetrans"]
        cc.internrot[1:nmt + 1], cc.interntrans[1:nmt + 1] = out["internrot"], out["interntrans"]
        cc.nmovei[1:3, 1:nmt + 1] = nmovei.reshape(2, nmt)
        if groups:
            cc.ninter[1:3, 1:nmt + 1] = d.m_ninter.cpu().numpy().reshape(2, nmt)
            cc.nstepreject[1:nmol + 1] = out["nstepreject"]
        self._coords_out()
        self._store_out(values_only=True)
        return out["fadds"], f32(fb.cpu().numpy()[0]), 1

    def en_change(self, im):
        """molfit.py:806-919 for molecule im (1-based) against its stored list; fills
        ergpairreference.ergnew and returns the energy change."""
        self._sync_in()
        self._store_in()
        d = self.d
        M = d.nnbrefmax
        erg = torch.zeros(max(M, 1), dtype=torch.float32, device=d.dev)
        out = np.zeros(1, f32)
        check(d.lib.epsr_en_change(C.byref(d.cbox), C.byref(d.store), int(im) - 1, C.c_void_p(erg.data_ptr()),
                                   out.ctypes.data_as(C.c_void_p), None))
        torch.cuda.synchronize()
        erd = self.c.ergpairreference
        n = int(erd.nergpairm[im])
        if n > 1:
            erd.ergnew[2:n + 1] = erg[1:n].cpu().numpy()
        return f32(out[0])

    def en_mole_pair(self, im, jm):
        """molfit.py:1528-1578: energy of molecules im and jm (1-based)."""
        self._sync_in()
        d = self.d
        ij = torch.tensor([int(im) - 1, int(jm) - 1], dtype=torch.int32, device=d.dev)
        res = torch.zeros(1, dtype=torch.float32, device=d.dev)
        check(d.lib.epsr_en_mole_pair(C.byref(d.cbox), C.c_void_p(ij.data_ptr()), C.c_void_p(ij.data_ptr() + 4), 1,
                                      C.c_void_p(res.data_ptr()), None))
        return f32(res.cpu().numpy()[0])

    def atogen(self, wav, ngrsamples):
        """ato_manipulation_rev4.py:3640-3899: fills wav(2,npt1,npairs) and potex in place;
        returns ngrsamples."""
        if self._outside_path():
            return self._host("atogen", wav, ngrsamples)
        c = self.c
        b = self._sync_in()
        pp = c.potential_par
        rminex = np.array([pp.rminex[int(pp.irefpcof[p + 1])] for p in range(b.npairs)], f32)
        t = self._ran1_in()
        n = self.d.atogen(int(ngrsamples), t, rminex, ycoh=np.asarray(c.epsr16.ycoh, f32),
                          sizefactor=f32(c.molecom.sizefactor))
        w, potex = self.d.download_wav()
        self._ran1_out(t)
        wav[1:3, 1:b.npt1 + 1, 1:b.npairs + 1] = w[:, :, 1:b.npt1 + 1].transpose(0, 2, 1)
        pp.potex[1:b.npairs + 1] = potex
        pp.potexmax[1:b.npairs + 1] = 0.0
        return n

    def press(self, energy, pressc, energf, pressf, energabs, energthreeb, prthreebout):
        """ato_manipulation_rev4.py:3903-4062: energy and pressure of the stored pairs on the
        device; abs_energy_ep and the per-file rescaling of energf/pressf (in place) on the
        host as the reference; returns (energy, pressc, energabs, energthreeb, prthreebout)."""
        if self._outside_path():
            return self._host("press", energy, pressc, energf, pressf, energabs, energthreeb, prthreebout)
        from .device import press_scalars
        c = self.c
        cc = c.clustercom
        b = self._sync_in()
        self._check_cells()
        self._store_in()
        energabs = self.mods["ato_manipulation_rev4"].abs_energy_ep()
        sumc, presst = self.d.press(int(c.epsr16.npt1), strict=self.strict)
        energy, pressc = press_scalars(b.nmol, sumc, presst, c.molecom.simt, cc.volume)
        nmol = f32(b.nmol)
        vol = f32(cc.volume)
        wsum = c.potential_par.wsum
        for i in range(1, int(c.epsr16.nfile) + 1):
            energf[i] = f32(energf[i]) / (nmol * f32(wsum[i]))
            pressf[i] = ((-f32(pressf[i]) / f32(3.0)) * f32(100.0)) / (f32(6.0222) * vol * f32(wsum[i]))
        return energy, pressc, energabs, f32(0.0), prthreebout

    def gensq(self, nq, q, sofq, wav):
        """epsr_standalone_rev3.py:4731-4802: fills sofq(2,nq,npairs) in place."""
        c = self.c
        if getattr(c.molecom_mod, "coarsegraining", False):
            return self._host("gensq", nq, q, sofq, wav)
        e16, mc = c.epsr16, c.molecom
        npairs, npt1, ntype = int(mc.npairs), int(e16.npt1), int(mc.ntype)
        ld = npt1 + 1
        w = np.ascontiguousarray(np.asarray(wav)[1:3, :ld, 1:npairs + 1].transpose(0, 2, 1), f32)
        fq = np.ascontiguousarray(np.asarray(e16.foqols)[:ld, :nq + 1], f32)
        out = transforms.gensq(int(nq), npt1, torch.from_numpy(w.reshape(-1)).cuda(), ld, fq, nq + 1, 1,
                               np.asarray(e16.ycoh[:ld], f32), np.asarray(mc.n2extr[1:npairs + 1], np.int32) - 1,
                               np.asarray(c.molecom_mod.natomsphere[1:ntype + 1], f32), npairs)
        o = out.cpu().numpy().reshape(2, npairs, nq + 1)
        sofq[1:3, 1:nq + 1, 1:npairs + 1] = o[:, :, 1:].transpose(0, 2, 1)
        return None

    def _running_sums(self, names, n, first, host_arrays, sample, call):
        """Upload the epsr16 accumulators (rows first..n of the reference's (point, pair)
        arrays), run `call` on them and the (2, points, pairs) sample on the device, write
        the rows back in place."""
        npairs = int(self.c.molecom.npairs)
        ld = n + 1
        acc = {k: torch.from_numpy(np.ascontiguousarray(np.asarray(host_arrays[k])[:ld, 1:npairs + 1].T, f32)).cuda()
               for k in names}
        w = np.ascontiguousarray(np.asarray(sample)[1:3, :ld, 1:npairs + 1].transpose(0, 2, 1), f32)
        call(torch.from_numpy(w.reshape(-1)).cuda(), acc)
        for k in names:
            host_arrays[k][first:ld, 1:npairs + 1] = acc[k].cpu().numpy()[:, first:ld].T
        return None

    def sumgr(self, nz, wav):
        """epsr_standalone_rev3.py:3578-3637: updates the running g(r) means, error bars and
        zero limits of epsr16 in place, with the weights fc1, fc2 of sumvalues."""
        c = self.c
        e16, sv = c.epsr16, c.sumvalues
        nz = int(nz)
        yc = torch.from_numpy(np.ascontiguousarray(np.asarray(e16.ycoh)[: nz + 1], f32)).cuda()
        arrays = {k: getattr(e16, k) for k in transforms.GR_ARRAYS}
        return self._running_sums(transforms.GR_ARRAYS, nz, 1, arrays, wav,
                                  lambda w, acc: transforms.sumgr(nz, w, yc, float(sv.fc1), float(sv.fc2), acc))

    def sumsq(self, nq, qwind):
        """epsr_standalone_rev3.py:3642-3677: updates the running S(Q) means and error bars
        of epsr16 in place."""
        c = self.c
        e16, sv = c.epsr16, c.sumvalues
        nq = int(nq)
        arrays = {k: getattr(e16, k) for k in transforms.SQ_ARRAYS}
        return self._running_sums(transforms.SQ_ARRAYS, nq, 1, arrays, qwind,
                                  lambda w, acc: transforms.sumsq(nq, w, float(sv.fc1), float(sv.fc2), acc))

    def generate_ep(self, changepotfac):
        """epsr_standalone_rev3.py:5876-6022: rebuilds xavs, xavs1, xavtot and xavtot1 of
        potential_par from the coefficients pcoefp, scales pcoefp by pressfac
        (multiply_pot_coeffs), and sets pwtold, expgr and (with changepotfac) potfac, in place.
        The basis matrix is built on the host once per grid and basis parameters."""
        from . import potential
        _lib.load(require_device=True)
        c = self.c
        pp, e16 = c.potential_par, c.epsr16
        npt, npt2, nterms = int(e16.npt), int(e16.npt2), int(pp.ncoeffp)
        npairs, nsets = int(c.molecom.npairs), int(pp.npairspcof)
        ld = npt + 1
        x = np.array(e16.x[:ld], f32)
        bp = (bool(pp.gaussian), f32(pp.pdmin), f32(pp.pdstep), f32(pp.pdmax), f32(pp.psigma2), f32(e16.rho),
              f32(c.epsrinput_par.rbroad))
        key = (npt2, nterms, *(float(v) for v in bp), x[: npt2 + 1].tobytes())
        cache = self._snap.get("ep_basis")
        if cache is None or cache[0] != key:
            expgr, _ = potential.basis(npt2, nterms, x, *bp)
            cache = (key, expgr, torch.from_numpy(expgr).cuda())
            self._snap["ep_basis"] = cache
        pp.expgr[1: npt2 * nterms + 1] = cache[1]
        dev = lambda a: torch.from_numpy(np.ascontiguousarray(a, f32)).cuda()  # noqa: E731
        tab = lambda a: dev(np.asarray(a)[:ld, 1:npairs + 1].T)  # noqa: E731
        tabs = {k: tab(getattr(pp, k)) for k in potential.TABLES}
        pc = dev(np.asarray(pp.pcoefp)[: nterms + 1, 1:nsets + 1].T)
        pw = dev(np.asarray(pp.pwtold)[: nterms + 1])
        pf = dev([pp.potfac])
        potential.generate_ep(npt, npt2, nterms, cache[2], pc, np.asarray(pp.irefpcof[1:npairs + 1], np.int32) - 1,
                              f32(c.clustercom.dmax), dev(np.asarray(e16.xstar)[:ld]), dev(np.asarray(pp.wfac)[:ld]),
                              tab(pp.ecoul), tabs, pw, f32(pp.absolute_energy), f32(pp.erequnit), f32(pp.ereqstep),
                              f32(pp.potfacamp), pf, bool(changepotfac))
        for k in potential.TABLES:
            getattr(pp, k)[1:ld, 1:npairs + 1] = tabs[k].cpu().numpy()[:, 1:ld].T
        pp.pcoefp[2: nterms + 1, 1:nsets + 1] = pc.cpu().numpy()[:, 2:].T
        pp.pwtold[1: nterms + 1] = pw.cpu().numpy()[1:]
        pp.potfac = f32(pf.cpu().numpy()[0])
        return None

    def generate_rp(self):
        """epsr_standalone_rev3.py:5675-5873 (generate_mp ato_manipulation_rev4.py:2816 first): the
        reference potential tables epot, epot1, ecoul, ecoul1, xav, xav1 of potential_par,
        rebuilt on the host by the library (the C library's float functions, as the reference)
        and written in place; the next device call uploads the changed tables.  Sets with
        container forces (rmaxex > 0) run the reference's own routine."""
        from . import potential
        c = self.c
        pp, mc, e16, ip = c.potential_par, c.molecom, c.epsr16, c.epsrinput_par
        npairs, npt, npt2 = int(mc.npairs), int(e16.npt), int(e16.npt2)
        iref = np.asarray(pp.irefpcof[1:npairs + 1], np.int32) - 1
        nsets = int(iref.max()) + 1
        if bool(np.any(np.asarray(pp.rmaxex[1:nsets + 1]) > 0.0)):
            return self._host("generate_rp")
        npg = np.asarray(pp.npgauss[1:nsets + 1], np.int32)
        maxg = max(1, int(npg.max()))
        g = lambda a: np.asarray(a)[1:maxg + 1, 1:nsets + 1].T  # noqa: E731
        ld = npt + 1
        out = potential.reference_potential(
            np.asarray(e16.x)[:ld], np.asarray(e16.xstar)[:ld], np.asarray(pp.wfac)[:ld], np.asarray(pp.wfacc)[:ld], npt,
            npt2, np.asarray(mc.n1extr[1:npairs + 1], np.int32) - 1, np.asarray(mc.n2extr[1:npairs + 1], np.int32) - 1,
            iref, np.asarray(mc.qradius)[1:], np.asarray(mc.ecor[1:npairs + 1]), np.asarray(mc.qcor[1:npairs + 1]),
            np.asarray(mc.dcor[1:npairs + 1]), np.asarray(pp.coulfac[1:nsets + 1]), np.asarray(pp.pcoefex[1:nsets + 1]),
            np.asarray(pp.rminex[1:nsets + 1]), mc.power, mc.ecore, mc.dcore, mc.sizefactor, pp.refpotfac, ip.expecf,
            ip.expecfpwr, bool(pp.harmonic), pp.addpotential == "modmorse", bool(mc.coul_intra), mc.coul_intra_fac, npg,
            g(pp.wpgauss), g(pp.rpgauss), g(pp.hpgauss))
        for k in potential.RP_TABLES:
            getattr(pp, k)[1:ld, 1:npairs + 1] = out[k][:, 1:ld].T
        return None

    def stog(self, rho, q, sofq, r, gofr, nqmin, nqmax, nr, npairs, nqdim, nrdim, npdim, xwt):
        """ato_manipulation_rev4.py:4067-4110: fills gofr(nr, npairs) in place."""
        ldq = int(nqdim) + 1
        qs = np.asarray(q[:ldq], f32)
        sp = np.ascontiguousarray(np.asarray(sofq)[:ldq, 1:npairs + 1].T, f32)
        g = transforms.stog(f32(rho), qs, torch.from_numpy(sp).cuda(), np.asarray(r[:nr + 1], f32),
                            np.asarray(nqmin[1:npairs + 1], np.int32), np.asarray(nqmax[1:npairs + 1], np.int32),
                            np.asarray(xwt[1:npairs + 1], f32))
        gofr[1:nr + 1, 1:npairs + 1] = g.cpu().numpy()[:, 1:nr + 1].T
        return None

    def fit_expansion(self, yin, expr, yout, wt, wtold, stepr, acceptr, rejrat, chisqnew, nmin, npt, ncfirst,
                      nterms, nits, nfreq):
        """epsr_standalone_rev3.py:4806-4921: fills wt, wtold, yout in place; returns
        (stepr, acceptr, rejrat, chisqnew)."""
        from .device import DeviceBox  # noqa: F401  (loads the library with a device check)
        _lib.load(require_device=True)
        r = self.c.ran1com
        st = Ran1State(idum=int(r.idum), iy=int(r.iy), mcall=int(np.int64(r.mcall) & 0xFFFFFFFF),
                       iv=np.asarray(r.iv[1:33], np.int32).copy())
        self._mcall0 = int(r.mcall)
        t = torch.from_numpy(st.as_array()).cuda()
        res = transforms.fit_expansion(np.asarray(yin[:npt + 1], f32), np.asarray(expr[:npt * nterms + 1], f32),
                                       np.asarray(wtold[:nterms + 1], f32), f32(stepr), int(nmin), int(npt),
                                       int(ncfirst), int(nterms), int(nits), int(nfreq), t, acceptr=f32(acceptr),
                                       rejrat=f32(rejrat), chisqnew=f32(chisqnew), strict=self.strict)
        self._ran1_out(t)
        wt[1:nterms + 1] = res["wt"].cpu().numpy()[1:nterms + 1]
        wtold[1:nterms + 1] = res["wtold"].cpu().numpy()[1:nterms + 1]
        yout[1:npt + 1] = res["yout"].cpu().numpy()[1:npt + 1]
        return res["stepr"], res["acceptr"], res["rejrat"], res["chisq"]


def install_reference(program, strict=False, routines=DEFAULT_ROUTINES):
    """Install the GPU path into a running reference process.

    ``program``: the loaded epsr program module (``epsr26.programs.load("epsr")``).  The
    library modules and the COMMON package are imported by name from ``epsr26``."""
    import importlib
    common = importlib.import_module("epsr26.common")
    mods = {"cellneighbourlist": importlib.import_module("epsr26.library.cellneighbourlist"),
            "ato_manipulation_rev4": importlib.import_module("epsr26.library.ato_manipulation_rev4"),
            "molfit": importlib.import_module("epsr26.library.molfit"), "program": program}
    for name in ("molecom", "clustercom", "epsr16", "potential_par", "lattice", "ran1com", "cellneighbourlist",
                 "ergpairreference", "molecom_mod", "threebody_mod", "coordconstraints_mod", "containerforces_mod"):
        importlib.import_module("epsr26.common." + name)
    return PairPath(common, mods, strict=strict).install(routines)
