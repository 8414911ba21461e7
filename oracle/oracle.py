"""ctypes wrapper of the C oracle (oracle/epsr_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by the tests, ``__graft_entry__.smoke()`` and the
CPU-baseline leg of ``bench.py`` as the checker.  The product library never loads it.

Functions take ``BoxArrays`` (epsr_python_translation_b200.box) and NumPy arrays and return
NumPy arrays laid out like the device path's outputs.
"""

from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "epsr_oracle.c")
LIB = os.path.join(HERE, "liboracle.so")

f32 = np.float32
P = C.c_void_p


def build(force=False):
    """Compile the restatement: float32 op order is kept by -ffp-contract=off."""
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(SRC):
        subprocess.check_call(["gcc", "-O2", "-fPIC", "-shared", "-ffp-contract=off", "-fno-fast-math",
                               "-o", LIB, SRC, "-lm"])
    return LIB


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        _lib = C.CDLL(LIB)
        _lib.oracle_ran1.restype = C.c_float
        _lib.oracle_en_mole_pair.restype = C.c_float
        _lib.oracle_fit_expansion.restype = C.c_int64
        _lib.oracle_fit_expansion_mode.restype = C.c_int64
    return _lib


def ptr(a):
    return a.ctypes.data_as(P) if a is not None else None


class Ran1C(C.Structure):
    _fields_ = [("idum", C.c_int32), ("iy", C.c_int32), ("mcall", C.c_int32), ("iv", C.c_int32 * 32)]

    @staticmethod
    def of(st):
        r = Ran1C()
        r.idum, r.iy, r.mcall = st.idum, st.iy, np.int64(st.mcall).astype(np.int32)
        for i in range(32):
            r.iv[i] = int(st.iv[i])
        return r

    def to_state(self):
        from epsr_python_translation_b200.box import Ran1State
        return Ran1State(self.idum, self.iy, self.mcall, np.array(list(self.iv), dtype=np.int32))


class SysC(C.Structure):
    _fields_ = [("nmol", C.c_int32), ("natom", C.c_int32), ("ntype", C.c_int32), ("npairs", C.c_int32),
                ("nmoltype", C.c_int32), ("naf", P), ("nato", P), ("mtype", P), ("itype", P),
                ("xa", P), ("ya", P), ("za", P), ("xadd", P), ("yadd", P), ("zadd", P), ("npairref", P),
                ("xstar", P), ("xavs", P), ("xavs1", P), ("ecoul", P), ("ecoul1", P), ("ld", C.c_int32),
                ("npt2", C.c_int32), ("stepcl", C.c_float), ("cubic", C.c_int32), ("lat", C.c_float * 6)]


class CellsC(C.Structure):
    _fields_ = [("ncelldiva", C.c_int32), ("ncelldivb", C.c_int32), ("ncelldivc", C.c_int32),
                ("ncell", C.c_int32), ("ncellneighb", C.c_int32), ("maxcellno", C.c_int32),
                ("molcellno", P), ("cell_start", P), ("cell_mols", P), ("ia_off", P), ("ib_off", P),
                ("ic_off", P)]


class StoreC(C.Structure):
    _fields_ = [("nnbrefmax", C.c_int32), ("nergpair", C.c_int32), ("nergpairmax", C.c_int32),
                ("nergpairm", P), ("molergpair", P), ("ergpairref", P), ("ergpair", P)]


class McParC(C.Structure):
    _fields_ = [("simt", C.c_float), ("rejrate", C.c_float), ("stepr", C.c_float), ("stepm", C.c_float),
                ("trstepmax", C.c_float), ("trstepmin", C.c_float), ("ireset", C.c_int32),
                ("wholerot", P), ("wholetrans", P), ("nwhole", P), ("nmovem", P), ("nstepreject", P),
                ("internrot", P), ("interntrans", P), ("ngrot", P)]


class TraceC(C.Structure):
    _fields_ = [("nmoves", C.c_int32), ("im", P), ("den", P), ("acc", P), ("cosv", P), ("ncos", C.c_int32),
                ("den64", P), ("scale64", P), ("u", P)]


class SysHandle:
    """Keeps the NumPy arrays alive for a SysC view of a BoxArrays (mutated in place)."""

    def __init__(self, box):
        self.box = box
        ld = box.npt + 1
        self.tabs = [np.ascontiguousarray(t, dtype=f32) for t in (box.xavs, box.xavs1, box.ecoul, box.ecoul1)]
        self.npairref = np.ascontiguousarray(box.npairref, dtype=np.int32)
        s = SysC()
        s.nmol, s.natom, s.ntype, s.npairs, s.nmoltype = box.nmol, box.natom, box.ntype, box.npairs, box.nmoltype
        s.naf, s.nato, s.mtype, s.itype = ptr(box.naf), ptr(box.nato), ptr(box.mtype), ptr(box.itype)
        s.xa, s.ya, s.za = ptr(box.xa), ptr(box.ya), ptr(box.za)
        s.xadd, s.yadd, s.zadd = ptr(box.xadd), ptr(box.yadd), ptr(box.zadd)
        s.npairref = ptr(self.npairref)
        s.xstar = ptr(box.xstar)
        s.xavs, s.xavs1, s.ecoul, s.ecoul1 = [ptr(t) for t in self.tabs]
        s.ld = ld
        s.npt2 = box.npt2
        s.stepcl = box.stepcl
        s.cubic = 1 if box.cubic else 0
        for i in range(6):
            s.lat[i] = float(box.lat6[i])
        self.c = s


# ----------------------------------------------------------------------------- ran1
def ran1_fill(state, n):
    r = Ran1C.of(state)
    out = np.zeros(n, dtype=f32)
    lib().oracle_ran1_fill(C.byref(r), ptr(out), C.c_int64(n))
    return out, r.to_state()


# ----------------------------------------------------------------------------- cells
def cell_list(box, nmolcell, rmax):
    L = lib()
    dims = np.zeros(4, dtype=np.int32)
    lat6 = np.ascontiguousarray(box.lat6, dtype=f32)
    lat9 = np.ascontiguousarray(box.lat9, dtype=f32)
    L.oracle_cell_dims(nmolcell, box.nmol, ptr(lat6), ptr(dims))
    ncell = int(dims[3])
    out = dict(molcellno=np.zeros(box.nmol, np.int32), cell_start=np.zeros(ncell + 1, np.int32),
               cell_mols=np.zeros(box.nmol, np.int32), ia_off=np.zeros(ncell, np.int32),
               ib_off=np.zeros(ncell, np.int32), ic_off=np.zeros(ncell, np.int32))
    c = CellsC()
    for k, v in out.items():
        setattr(c, k, ptr(v))
    L.oracle_cell_list(nmolcell, ptr(box.xadd), ptr(box.yadd), ptr(box.zadd), box.nmol, C.c_float(f32(rmax)),
                       ptr(lat6), ptr(lat9), C.byref(c))
    out.update(ncelldiva=c.ncelldiva, ncelldivb=c.ncelldivb, ncelldivc=c.ncelldivc, ncell=c.ncell,
               ncellneighb=c.ncellneighb, maxcellno=c.maxcellno)
    out["_keep"] = [out[k] for k in ("molcellno", "cell_start", "cell_mols", "ia_off", "ib_off", "ic_off")]
    for k in ("ia_off", "ib_off", "ic_off"):
        out[k] = out[k][: c.ncellneighb].copy()
    out["_c"] = c
    out["nnbrefmax"] = int(L.oracle_nnbrefmax(C.byref(c)))
    return out


def cells_from_arrays(dims, cell_start, cell_mols, molcellno, offsets, nnbrefmax):
    """A cell list given as arrays (the reference's own, read from its COMMON block): dims =
    (ncelldiva, ncelldivb, ncelldivc, ncell, ncellneighb, maxcellno), cell_start (ncell+1),
    cell_mols (0-based molecules in cell order), molcellno (1-based), offsets (ncellneighb x 3)."""
    ncell, nb = int(dims[3]), int(dims[4])
    noff = max(ncell, nb)
    out = dict(molcellno=np.ascontiguousarray(molcellno, np.int32), cell_start=np.ascontiguousarray(cell_start, np.int32),
               cell_mols=np.ascontiguousarray(cell_mols, np.int32), ia_off=np.zeros(noff, np.int32),
               ib_off=np.zeros(noff, np.int32), ic_off=np.zeros(noff, np.int32))
    for i, k in enumerate(("ia_off", "ib_off", "ic_off")):
        out[k][:nb] = np.asarray(offsets)[:, i]
    c = CellsC()
    for k in ("molcellno", "cell_start", "cell_mols", "ia_off", "ib_off", "ic_off"):
        setattr(c, k, ptr(out[k]))
    c.ncelldiva, c.ncelldivb, c.ncelldivc, c.ncell, c.ncellneighb, c.maxcellno = (int(v) for v in dims)
    out["_keep"] = [out[k] for k in ("molcellno", "cell_start", "cell_mols", "ia_off", "ib_off", "ic_off")]
    out["_c"] = c
    out["nnbrefmax"] = int(nnbrefmax)
    out.update(ncelldiva=c.ncelldiva, ncelldivb=c.ncelldivb, ncelldivc=c.ncelldivc, ncell=ncell, ncellneighb=nb,
               maxcellno=c.maxcellno)
    return out


def region(cells, ic):
    nb = np.zeros(max(cells["nnbrefmax"], 1), dtype=np.int32)
    n = lib().oracle_region(C.byref(cells["_c"]), ic, ptr(nb))
    return nb[:n].copy()


# ----------------------------------------------------------------------------- fmolec1
def fmolec1(box, cells, eintra, capacity=None):
    M = cells["nnbrefmax"]
    nmol = box.nmol
    cap = capacity or 100 * nmol
    while True:
        st = dict(nergpairm=np.zeros(nmol, np.int32), molergpair=np.zeros(nmol * M, np.int32),
                  ergpairref=np.zeros(nmol * M, np.int32), ergpair=np.zeros(cap, f32))
        E = StoreC()
        E.nnbrefmax, E.nergpair, E.nergpairmax = M, 0, cap
        for k, v in st.items():
            setattr(E, k, ptr(v))
        out2 = np.zeros(2, f32)
        h = SysHandle(box)
        ei = np.ascontiguousarray(eintra, dtype=f32)
        rc = lib().oracle_fmolec1(C.byref(h.c), C.byref(cells["_c"]), ptr(ei), C.byref(E), ptr(out2))
        if rc == 0:
            break
        cap = cap * 2
    st["molergpair"] = st["molergpair"].reshape(nmol, M)
    st["ergpairref"] = st["ergpairref"].reshape(nmol, M)
    st["nergpair"] = E.nergpair
    st["nnbrefmax"] = M
    st["ftest"] = out2[0]
    st["ftestb"] = out2[1]
    st["_cap"] = cap
    return st


def store_c(st):
    E = StoreC()
    E.nnbrefmax, E.nergpair, E.nergpairmax = st["nnbrefmax"], st["nergpair"], st["ergpair"].shape[0]
    E.nergpairm = ptr(st["nergpairm"])
    E.molergpair = ptr(st["molergpair"])
    E.ergpairref = ptr(st["ergpairref"])
    E.ergpair = ptr(st["ergpair"])
    return E


def en_mole_pair(box, im, jm):
    h = SysHandle(box)
    return f32(lib().oracle_en_mole_pair(C.byref(h.c), int(im), int(jm)))


# ----------------------------------------------------------------------------- press
def press_scalars(nmol, sumc, presst, simt, volume):
    """The closing lines of press (ato_manipulation_rev4.py:4051-4056): energy per molecule
    (float32) and pressure in kbar (double arithmetic, stored as float32)."""
    energy = f32(f32(sumc) / f32(nmol))
    pressc = f32(((float(f32(nmol) * f32(simt)) - float(presst) / 3.0) * 100.0)
                 / float(f32(6.0222) * f32(volume)))
    return energy, pressc


def press_file_terms(nmol, energf, pressf, wsum, volume):
    """Per-file rescaling at the end of press (:4057-4060), float32."""
    ef = f32(energf) / (f32(nmol) * f32(wsum))
    pf = ((-f32(pressf) / f32(3.0)) * f32(100.0)) / (f32(6.0222) * f32(volume) * f32(wsum))
    return f32(ef), f32(pf)


def press(box, st, npt1, simt, volume):
    """press on the stored pairs (no three-body or coordination terms): returns sumc,
    presst, the double sum of the same float32 pair energies (sum64) and the energy and
    pressure the reference returns."""
    h = SysHandle(box)
    E = store_c(st)
    L = lib()
    L.oracle_press.restype = C.c_float
    d = np.zeros(2, np.float64)
    sumc = f32(L.oracle_press(C.byref(h.c), C.byref(E), int(npt1), ptr(d)))
    energy, pressc = press_scalars(box.nmol, sumc, d[0], simt, volume)
    return dict(sumc=sumc, presst=float(d[0]), sum64=float(d[1]), energy=energy, pressc=pressc)


# ----------------------------------------------------------------------------- molfit
def trsteps(natomr):
    out = np.zeros(2, f32)
    lib().oracle_trsteps(natomr, ptr(out))
    return out[0], out[1]


class RotC(C.Structure):
    _fields_ = [("I", P), ("nrf", P), ("nrl", P), ("axis", P), ("first", P), ("last", P), ("atoms", P),
                ("stepri", C.c_float), ("rotcycle", C.c_int32), ("ninter", P), ("faddbs", P)]


def molfit(box, cells, st, mc, ran1, fadds=0.0, record_cos=True, rot=None):
    """One whole-molecule cycle; mutates box coordinates, st['ergpair'] and the step arrays
    in ``mc`` (dict of NumPy arrays).  Returns (fadds, trace dict, ran1 state).  ``rot``: the
    internal rotations of rotational groups (type ROT) before each molecule's move, a dict with
    model (the intramolecular model of molfit_shake, its ngrot included), nrf, nrl (per
    molecule), axis (groups x 2), first, last (per group, into atoms), atoms (0-based), stepri,
    rotcycle and faddbs; the trace then also holds ninter (2*nmoltype) and faddbs."""
    h = SysHandle(box)
    E = store_c(st)
    nmt = box.nmoltype
    par = McParC()
    par.simt, par.rejrate = box.simt, f32(mc["rejrate"])
    par.stepr, par.stepm = f32(mc["stepr"]), f32(mc["stepm"])
    tmax, tmin = trsteps(box.natomr)
    par.trstepmax, par.trstepmin = tmax, tmin
    par.ireset = int(mc.get("ireset", 0))
    for k in ("wholerot", "wholetrans", "internrot", "interntrans"):
        mc[k] = np.ascontiguousarray(mc[k], dtype=f32)
        setattr(par, k, ptr(mc[k]))
    mc["nwhole"] = np.zeros(2 * nmt, np.int32)
    mc["nmovem"] = np.zeros(2 * nmt, np.int32)
    mc["nstepreject"] = np.ascontiguousarray(mc.get("nstepreject", np.zeros(box.nmol, np.int32)), np.int32)
    mc["ngrot"] = np.ascontiguousarray(mc.get("ngrot", np.zeros(box.nmol, np.int32)), np.int32)
    par.nwhole, par.nmovem = ptr(mc["nwhole"]), ptr(mc["nmovem"])
    par.nstepreject, par.ngrot = ptr(mc["nstepreject"]), ptr(mc["ngrot"])
    tr = dict(im=np.zeros(box.nmol, np.int32), den=np.zeros(box.nmol, f32), acc=np.zeros(box.nmol, np.int32),
              cosv=np.zeros(3 * box.nmol, f32) if record_cos else None,
              den64=np.zeros(box.nmol, np.float64), scale64=np.zeros(box.nmol, np.float64),
              u=np.zeros(box.nmol, f32))
    T = TraceC()
    T.den64, T.scale64, T.u = ptr(tr["den64"]), ptr(tr["scale64"]), ptr(tr["u"])
    T.im, T.den, T.acc = ptr(tr["im"]), ptr(tr["den"]), ptr(tr["acc"])
    T.cosv = ptr(tr["cosv"]) if record_cos else None
    r = Ran1C.of(ran1)
    fa = C.c_float(f32(fadds))
    if rot is None:
        lib().oracle_molfit(C.byref(h.c), C.byref(cells["_c"]), C.byref(E), C.byref(par), C.byref(r), C.byref(fa),
                            C.byref(T))
    else:
        T.cosv = ptr(tr["cosv"]) if record_cos else None
        if record_cos:
            tr["cosv"] = np.zeros(3 * box.nmol + int(np.asarray(rot["first"]).size) * box.nmol, f32)
            T.cosv = ptr(tr["cosv"])
        ih = IntraHandle(box, rot["model"])
        arrs = {k: np.ascontiguousarray(rot[k], np.int32) for k in ("nrf", "nrl", "axis", "first", "last", "atoms")}
        ninter = np.zeros(2 * nmt, np.int32)
        fb = np.array([f32(rot.get("faddbs", 0.0))], f32)
        rc = RotC()
        rc.I = C.cast(C.pointer(ih.c), P)
        for k, v in arrs.items():
            setattr(rc, k, ptr(v))
        rc.stepri, rc.rotcycle = f32(rot["stepri"]), int(rot["rotcycle"])
        rc.ninter, rc.faddbs = ptr(ninter), ptr(fb)
        lib().oracle_molfit_rot(C.byref(h.c), C.byref(cells["_c"]), C.byref(E), C.byref(par), C.byref(r),
                                C.byref(fa), C.byref(T), C.byref(rc))
        tr["ninter"] = ninter
        tr["faddbs"] = f32(fb[0])
    tr["nmoves"] = T.nmoves
    if record_cos:
        tr["cosv"] = tr["cosv"][: T.ncos].copy()
    return f32(fa.value), tr, r.to_state()


# ----------------------------------------------------------------------------- intramolecular
class IntraC(C.Structure):
    _fields_ = [("nbond", P), ("iabond", P), ("tbond", P), ("maxbond", C.c_int32), ("imageatom", P), ("qtype", P),
                ("amassa", P), ("amassr", P), ("xav", P), ("xav1", P), ("ngrot", P), ("stepcl", C.c_float),
                ("sizefactor", C.c_float), ("tempb", C.c_float), ("tempang", C.c_float), ("simt", C.c_float),
                ("refine_intra", C.c_int32), ("refine_intra_fac", C.c_float), ("ndih", C.c_int32), ("grp_nrf", P),
                ("grp_nrl", P), ("grp_axis", P), ("grp_dih0", P), ("grp_isdih", P), ("dih_atoms", P), ("dih_cos", P),
                ("dih_sin", P), ("tempdih", C.c_float)]


class IntraHandle:
    """Keeps the NumPy arrays of an intramolecular model alive for its IntraC view.  ``m``: dict
    with nbond (natom,), iabond/tbond (natom, maxbond) 0-based, amassa, amassr, xav/xav1
    (npairs, ld), stepcl, sizefactor, tempb, tempang, simt, refine_intra, refine_intra_fac and
    optional imageatom/qtype/ngrot; optional ``dih``: the rotational groups' dihedral angles, a
    dict with grp_nrf, grp_nrl (per molecule, 0-based), grp_axis (groups x 2), grp_dih0
    (groups + 1), grp_isdih (groups), dih_atoms (dihedrals x 2), dih_cos, dih_sin, tempdih."""

    def __init__(self, box, m):
        self.a = dict(nbond=np.ascontiguousarray(m["nbond"], np.int32),
                      iabond=np.ascontiguousarray(m["iabond"], np.int32),
                      tbond=np.ascontiguousarray(m["tbond"], f32),
                      imageatom=np.ascontiguousarray(m.get("imageatom", np.full(box.natom, -1)), np.int32),
                      qtype=np.ascontiguousarray(m.get("qtype", np.zeros(box.natom)), np.int32),
                      amassa=np.ascontiguousarray(m["amassa"], f32), amassr=np.ascontiguousarray(m["amassr"], f32),
                      xav=np.ascontiguousarray(m["xav"], f32), xav1=np.ascontiguousarray(m["xav1"], f32),
                      ngrot=np.ascontiguousarray(m.get("ngrot", np.zeros(box.nmol)), np.int32))
        c = IntraC()
        for k, v in self.a.items():
            setattr(c, k, ptr(v))
        c.maxbond = self.a["iabond"].shape[1]
        for k in ("stepcl", "sizefactor", "tempb", "tempang", "simt", "refine_intra_fac"):
            setattr(c, k, f32(m[k]))
        c.refine_intra = int(bool(m["refine_intra"]))
        dh = m.get("dih")
        if dh is not None:
            for k in ("grp_nrf", "grp_nrl", "grp_axis", "grp_dih0", "grp_isdih", "dih_atoms"):
                self.a[k] = np.ascontiguousarray(dh[k], np.int32).reshape(-1)
                setattr(c, k, ptr(self.a[k]))
            for k in ("dih_cos", "dih_sin"):
                self.a[k] = np.ascontiguousarray(dh[k], f32)
                setattr(c, k, ptr(self.a[k]))
            c.ndih = int(self.a["dih_cos"].size)
            c.tempdih = f32(dh["tempdih"])
        self.c = c


def minimage_centres(box):
    """runepsr17 epsr_standalone_rev3.py:1332-1335 (minimagec of every centre), in place."""
    h = SysHandle(box)
    lib().oracle_minimage_centres(C.byref(h.c))


def en_mole_intra_all(box, m):
    """en_mole_intra molfit.py:1327-1350 of every molecule (C restatement)."""
    h, ih = SysHandle(box), IntraHandle(box, m)
    out = np.zeros(box.nmol, f32)
    lib().oracle_en_mole_intra_all(C.byref(h.c), C.byref(ih.c), ptr(out))
    return out


def molfit_shake(box, st, mc, m, stepmi, ran1, fadds, faddbs, ergold1=0.0):
    """The intramolecular cycle of molfit (molfit.py:119-174, :246-247, then :465-536), C
    restatement.  Mutates the box coordinates, st["ergpair"] and the step arrays in ``mc``.
    Returns (fadds, faddbs, nmovei (2*nmt,), ergold1, ran1 state)."""
    h, ih = SysHandle(box), IntraHandle(box, m)
    E = store_c(st)
    nmt = box.nmoltype
    par = McParC()
    par.simt, par.rejrate = box.simt, f32(mc["rejrate"])
    tmax, tmin = trsteps(box.natomr)
    par.trstepmax, par.trstepmin = tmax, tmin
    par.ireset = int(mc.get("ireset", 0))
    for k in ("wholerot", "wholetrans", "internrot", "interntrans"):
        mc[k] = np.ascontiguousarray(mc[k], dtype=f32)
        setattr(par, k, ptr(mc[k]))
    mc["nwhole"] = np.zeros(2 * nmt, np.int32)
    mc["nmovem"] = np.zeros(2 * nmt, np.int32)
    par.nwhole, par.nmovem = ptr(mc["nwhole"]), ptr(mc["nmovem"])
    nmovei = np.zeros(2 * nmt, np.int32)
    r = Ran1C.of(ran1)
    fa, fb, eo = C.c_float(f32(fadds)), C.c_float(f32(faddbs)), C.c_float(f32(ergold1))
    rc = lib().oracle_molfit_shake(C.byref(h.c), C.byref(E), C.byref(par), C.byref(ih.c), C.c_float(f32(stepmi)),
                                   C.byref(r), C.byref(fa), C.byref(fb), ptr(nmovei), C.byref(eo))
    if rc:
        raise ValueError("molfit_shake: molecules with rotational groups")
    return f32(fa.value), f32(fb.value), nmovei, f32(eo.value), r.to_state()


def molfit_shake_rot(box, st, mc, rot, stepmi, ran1, fadds, faddbs, ergold1=0.0):
    """The intramolecular cycle of molfit for a box with ROT groups (molfit.py:124-267: random
    atom moves, then the internal rotations tested with the intermolecular change; step
    adaptation :465-536), C restatement.  ``rot`` as for molfit (model, nrf, nrl, axis, first,
    last, atoms, stepri); ``mc`` holds ngrot and nstepreject besides the step arrays.  Mutates
    the box coordinates, st["ergpair"] and ``mc``.  Returns (fadds, faddbs, nmovei (2*nmt,),
    ninter (2*nmt,), ergold1, ran1 state, the cosines rotati drew)."""
    h, ih = SysHandle(box), IntraHandle(box, rot["model"])
    E = store_c(st)
    nmt = box.nmoltype
    par = McParC()
    par.simt, par.rejrate = box.simt, f32(mc["rejrate"])
    tmax, tmin = trsteps(box.natomr)
    par.trstepmax, par.trstepmin = tmax, tmin
    par.ireset = int(mc.get("ireset", 0))
    for k in ("wholerot", "wholetrans", "internrot", "interntrans"):
        mc[k] = np.ascontiguousarray(mc[k], dtype=f32)
        setattr(par, k, ptr(mc[k]))
    mc["nwhole"] = np.zeros(2 * nmt, np.int32)
    mc["nmovem"] = np.zeros(2 * nmt, np.int32)
    mc["nstepreject"] = np.ascontiguousarray(mc.get("nstepreject", np.zeros(box.nmol, np.int32)), np.int32)
    mc["ngrot"] = np.ascontiguousarray(mc["ngrot"], np.int32)
    par.nwhole, par.nmovem = ptr(mc["nwhole"]), ptr(mc["nmovem"])
    par.nstepreject, par.ngrot = ptr(mc["nstepreject"]), ptr(mc["ngrot"])
    arrs = {k: np.ascontiguousarray(rot[k], np.int32) for k in ("nrf", "nrl", "axis", "first", "last", "atoms")}
    ninter = np.zeros(2 * nmt, np.int32)
    rc = RotC()
    rc.I = C.cast(C.pointer(ih.c), P)
    for k, v in arrs.items():
        setattr(rc, k, ptr(v))
    rc.stepri, rc.rotcycle, rc.ninter, rc.faddbs = f32(rot["stepri"]), 1, ptr(ninter), None
    cosv = np.zeros(int(arrs["first"].size) + 1, f32)
    T = TraceC()
    T.cosv = ptr(cosv)
    nmovei = np.zeros(2 * nmt, np.int32)
    r = Ran1C.of(ran1)
    fa, fb, eo = C.c_float(f32(fadds)), C.c_float(f32(faddbs)), C.c_float(f32(ergold1))
    if lib().oracle_molfit_shake_rot(C.byref(h.c), C.byref(E), C.byref(par), C.byref(rc), C.c_float(f32(stepmi)),
                                     C.byref(r), C.byref(fa), C.byref(fb), ptr(nmovei), C.byref(eo), C.byref(T)):
        raise ValueError("molfit_shake_rot: a molecule of more than 4096 atoms")
    return f32(fa.value), f32(fb.value), nmovei, ninter, f32(eo.value), r.to_state(), cosv[: T.ncos].copy()


# ----------------------------------------------------------------------------- atogen
def atogen(box, ngrsamples, ran1, rminex, ycoh=None, sizefactor=1.0):
    ld = box.npt + 1
    wav = np.zeros((2, box.npairs, ld), f32)
    potex = np.zeros(box.npairs, f32)
    if ycoh is None:
        ycoh = np.zeros(ld, f32)
    ycoh = np.ascontiguousarray(ycoh[:ld], dtype=f32)
    h = SysHandle(box)
    r = Ran1C.of(ran1)
    rmx = np.ascontiguousarray(rminex, dtype=f32)
    ngr = lib().oracle_atogen(C.byref(h.c), ptr(wav), ptr(potex), int(ngrsamples), int(box.npt1),
                              C.c_float(f32(sizefactor)), C.c_float(f32(box.dmax)), ptr(rmx), ptr(box.cfrac),
                              int(box.natomr), ptr(ycoh), C.byref(r))
    return wav, potex, int(ngr), r.to_state()


# ----------------------------------------------------------------------------- transforms
def ptgnsq_difference(data, cwt, qwind, q=None, nqmin=None, nqmax=None, szeros=None, qmin=0.0, wq=None, xray=None):
    """ptgnsq epsr_standalone_rev3.py:3844-3867: the simulated fit of data set d at Q index i
    is the sum over atom pairs ic, in order, of cwt[d, ic] * qwind[ic, i] (:3853-3854); the
    weights are real*8 (weights.py:23), so each step is sum = real(dble(sum) + cwt *
    dble(qwind)): product and sum in double, one rounding to float32.  Returned negated as
    the difference from the data, -qtemp, with the Q window of :3856-3867 when q is given
    (per data set nqmin, nqmax, szeros; qmin the reference's qminptemp)."""
    data = np.asarray(data, np.float32)
    cwt = np.asarray(cwt, np.float64)
    qwind = np.asarray(qwind, np.float32)
    out = np.empty_like(data)
    for d in range(data.shape[0]):
        s = np.zeros(qwind.shape[1], np.float32)
        xr = wq is not None and xray is not None and int(xray[d]) != 0   # x_rayf0.weightx (:3850-3852)
        for ic in range(qwind.shape[0]):
            w = np.asarray(wq[d, ic], np.float64) if xr else cwt[d, ic]
            s = (s.astype(np.float64) + w * qwind[ic].astype(np.float64)).astype(np.float32)
        if q is None:
            out[d] = -(data[d] - s)
            continue
        f = np.float32
        nq = data.shape[1] - 1
        nqmn = 1 if nqmin is None else int(nqmin[d])
        nqmx = nq if nqmax is None else int(nqmax[d])
        sz = f(0.0) if szeros is None else f(szeros[d])
        qq = np.asarray(q, f)
        grads0 = conss0 = f(0.0)
        if sz != 0.0 and nqmn > 1:
            grads0 = f(f(data[d, nqmn] - sz) / f(qq[nqmn] - qq[1]))
            conss0 = sz
        qthr = qq[nqmn] if qq[nqmn] > f(qmin) else f(qmin)
        for i in range(nq + 1):
            if qq[i] < qthr:
                qt = f(f(conss0 + f(grads0 * f(qq[i] - qq[1]))) - s[i]) if sz != 0.0 else f(0.0)
            elif nqmn <= i <= nqmx:
                qt = f(data[d, i] - s[i])
            else:
                qt = f(0.0)
            out[d, i] = -qt
    return out


def gensq(nq, npt1, wav, foqols_rows, ycoh, n2extr, natomsphere):
    """wav (2, npairs, ldw); foqols_rows (nq+1, ldf) with row i = F[:, i]."""
    npairs, ldw = wav.shape[1], wav.shape[2]
    ldf = foqols_rows.shape[1]
    out = np.zeros((2, npairs, nq + 1), f32)
    lib().oracle_gensq(nq, npairs, npt1, ptr(np.ascontiguousarray(wav, f32)), ldw,
                       ptr(np.ascontiguousarray(foqols_rows, f32)), ldf, ptr(np.ascontiguousarray(ycoh, f32)),
                       ptr(np.ascontiguousarray(n2extr, np.int32)), ptr(np.ascontiguousarray(natomsphere, f32)),
                       ptr(out))
    return out


def sumgr(nz, wav, ycoh, fc1, fc2, acc):
    """sumgr epsr_standalone_rev3.py:3578-3637 (C restatement).  wav (2, npairs, ldw); acc a
    dict of (npairs, ldw) float32 arrays gorintra, gorinter, gr2intra, gr2inter, entsig,
    returned updated (copies)."""
    npairs, ldw = wav.shape[1], wav.shape[2]
    out = {k: np.ascontiguousarray(acc[k], f32).copy() for k in ("gorintra", "gorinter", "gr2intra", "gr2inter",
                                                                  "entsig")}
    lib().oracle_sumgr(int(nz), npairs, ptr(np.ascontiguousarray(wav, f32)), ldw, ptr(np.ascontiguousarray(ycoh, f32)),
                       C.c_double(fc1), C.c_double(fc2), ptr(out["gorintra"]), ptr(out["gorinter"]),
                       ptr(out["gr2intra"]), ptr(out["gr2inter"]), ptr(out["entsig"]))
    return out


def sumsq(nq, qwind, fc1, fc2, acc):
    """sumsq epsr_standalone_rev3.py:3642-3677 (C restatement).  qwind (2, npairs, ldq); acc a
    dict of (npairs, ldq) float32 arrays soqintra, soqinter, sq2intra, sq2inter."""
    npairs, ldq = qwind.shape[1], qwind.shape[2]
    out = {k: np.ascontiguousarray(acc[k], f32).copy() for k in ("soqintra", "soqinter", "sq2intra", "sq2inter")}
    lib().oracle_sumsq(int(nq), npairs, ptr(np.ascontiguousarray(qwind, f32)), ldq, C.c_double(fc1),
                       C.c_double(fc2), ptr(out["soqintra"]), ptr(out["soqinter"]), ptr(out["sq2intra"]),
                       ptr(out["sq2inter"]))
    return out


def generate_ep(npt, npt2, nterms, expgr, pcoefp, iref, dmax, xstar, wfac, ecoul, tabs, pwtold, par, potfac,
                changepotfac=True):
    """generate_ep epsr_standalone_rev3.py:5876-6022 (C restatement) from the basis matrix
    expgr (npt2*nterms,) the reference's calc_pwrexpr_grad builds.  pcoefp (nsets, ldc >=
    nterms+1) [set, ic]; iref (npairs,) 0-based set of each pair; ecoul and tabs["xavs", "xavs1",
    "xavtot", "xavtot1"] (npairs, ld) [pair, j]; pwtold (nterms+1,); par (absolute_energy,
    erequnit, ereqstep, potfacamp).  Returns (tabs, pcoefp, pwtold, potfac, energabs,
    pressfac), all updated copies."""
    npairs, ld = ecoul.shape
    nsets = pcoefp.shape[0]
    pc = np.ascontiguousarray(pcoefp, f32).copy()
    out = {k: np.ascontiguousarray(tabs[k], f32).copy() for k in ("xavs", "xavs1", "xavtot", "xavtot1")}
    pw = np.ascontiguousarray(pwtold, f32).copy()
    pf = np.array([potfac], f32)
    o2 = np.zeros(2, f32)
    lib().oracle_generate_ep(npairs, int(npt), int(npt2), int(nterms), ptr(np.ascontiguousarray(expgr, f32)), ptr(pc),
                             nsets, pc.shape[1], ptr(np.ascontiguousarray(iref, np.int32)), C.c_float(f32(dmax)),
                             ptr(np.ascontiguousarray(xstar, f32)), ptr(np.ascontiguousarray(wfac, f32)),
                             ptr(np.ascontiguousarray(ecoul, f32)), ptr(out["xavs"]), ptr(out["xavs1"]),
                             ptr(out["xavtot"]), ptr(out["xavtot1"]), ld, ptr(pw), ptr(np.ascontiguousarray(par, f32)),
                             ptr(pf), int(bool(changepotfac)), ptr(o2))
    return out, pc, pw, pf[0], o2[0], o2[1]


def calc_pwrexpr_grad(lpt, nterms, dmin, dstep, dmax, sigmab, rho, x, rmin=0.0, fbroad=1.0, rbroad=0.0):
    """calc_pwrexpr_grad epsr_standalone_rev3.py:5230-5309 (C restatement): the r-space basis
    (lpt*nterms,) on x[1..lpt] (x 1-based)."""
    out = np.zeros(int(lpt) * int(nterms), f32)
    nc = lib().oracle_calc_pwrexpr_grad(int(lpt), int(nterms), C.c_float(f32(dmin)), C.c_float(f32(dstep)),
                                        C.c_float(f32(dmax)), C.c_float(f32(sigmab)), C.c_float(f32(rho)),
                                        ptr(np.ascontiguousarray(x, f32)), ptr(out), C.c_float(f32(rmin)), 0,
                                        C.c_float(f32(fbroad)), C.c_float(f32(rbroad)))
    if nc < 0:
        raise IndexError("calc_pwrexpr_grad: log-factorial table too short")
    return out


def ep_update(pcoefp, iref, efacp, cwtpot, pwtold, pfact):
    """ptgnsq's coefficient increment epsr_standalone_rev3.py:3948-3962, per data set id in
    turn: pcoefp(ic, k) = real(dble(pcoefp) + (dble(pfact * efacp(k)) * cwtpot(ip, id)) *
    dble(pwtold_id(ic))) for ic = 2..nterms and every pair ip (set k = iref[ip]) in order;
    cwtpot is real*8 (weights.py:25), so each increment is formed in double and rounded once.
    pcoefp (nsets, ldc) [set, ic]; cwtpot (ndata, npairs); pwtold (ndata, nterms+1).
    Returns an updated copy."""
    pc = np.array(pcoefp, f32)
    pfact = f32(pfact)
    nterms = pwtold.shape[1] - 1
    cw = np.asarray(cwtpot, np.float64)
    for d in range(cw.shape[0]):
        pw = np.asarray(pwtold[d, 2: nterms + 1], f32).astype(np.float64)
        for ip, k in enumerate(np.asarray(iref)):
            fk = float(f32(pfact * f32(efacp[k])))
            pc[k, 2: nterms + 1] = (pc[k, 2: nterms + 1].astype(np.float64) + (fk * cw[d, ip]) * pw).astype(f32)
    return pc


def stog(rho, q, sofq_pairs, r, nqmin, nqmax, xwt):
    """q (ldq,), sofq_pairs (npairs, ldq) 1-based i; r (nr+1,) 1-based. Returns (npairs, nr+1)."""
    npairs, ldq = sofq_pairs.shape
    nr = r.shape[0] - 1
    out = np.zeros((npairs, nr + 1), f32)
    lib().oracle_stog(C.c_float(f32(rho)), ptr(np.ascontiguousarray(q, f32)),
                      ptr(np.ascontiguousarray(sofq_pairs, f32)), ldq, ptr(np.ascontiguousarray(r, f32)), ptr(out),
                      ptr(np.ascontiguousarray(nqmin, np.int32)), ptr(np.ascontiguousarray(nqmax, np.int32)), nr,
                      npairs, ptr(np.ascontiguousarray(xwt, f32)))
    return out


def fit_expansion(yin, expr, wtold, stepr, nmin, npt, ncfirst, nterms, nits, nfreq, ran1, fast=False, acceptr=0.0,
                  rejrat=0.0, chisqnew=0.0):
    """1-based arrays (index 0 unused).  Returns dict and the new ran1 state.  fast: the trial
    loop's chi^2 summed in double and rounded once to float32 (the device's fast mode); the
    final chi^2 keeps the reference's sequential float sum in both modes.  acceptr, rejrat,
    chisqnew: the caller's values of the in/out arguments (epsr_standalone_rev3.py:4806)."""
    yin = np.ascontiguousarray(yin, f32)
    expr = np.ascontiguousarray(expr, f32)
    wt = np.zeros(nterms + 1, f32)
    wto = np.ascontiguousarray(wtold, f32).copy()
    yout = np.zeros(npt + 1, f32)
    scal = np.array([stepr, acceptr, rejrat, chisqnew], f32)
    r = Ran1C.of(ran1)
    trials = lib().oracle_fit_expansion_mode(ptr(yin), ptr(expr), ptr(yout), ptr(wt), ptr(wto), ptr(scal), nmin,
                                             npt, ncfirst, nterms, nits, nfreq, C.byref(r), 1 if fast else 0)
    return dict(wt=wt, wtold=wto, yout=yout, stepr=scal[0], acceptr=scal[1], rejrat=scal[2], chisq=scal[3],
                trials=int(trials)), r.to_state()


def en_change(box, st, im):
    """en_change at the current coordinates: (float32 value, exact double sum of the same
    terms, sum of their magnitudes, ergnew)."""
    L = lib()
    L.oracle_en_change.restype = C.c_float
    h = SysHandle(box)
    E = store_c(st)
    ergnew = np.zeros(max(st["nnbrefmax"], 1), f32)
    d = np.zeros(2, np.float64)
    v = L.oracle_en_change(C.byref(h.c), int(im), C.byref(E), ptr(ergnew), ptr(d))
    return f32(v), float(d[0]), float(d[1]), ergnew


def en_mole_pair64(box, im, jm):
    """FP64 en_mole_pair: (energy, sum of |atom-pair terms|)."""
    h = SysHandle(box)
    out = np.zeros(2, np.float64)
    lib().oracle_en_mole_pair64(C.byref(h.c), int(im), int(jm), ptr(out))
    return float(out[0]), float(out[1])
