"""Golden vectors for the internal rotations of rotational groups in molfit's whole-molecule
cycle (molfit.py:295-360, rotati :589), made by running the reference translation (epsr26).

    EPSR_REFERENCE=<reference checkout> PYTHONDONTWRITEBYTECODE=1 python tests/golden/make_golden_rot.py

A 20 DMSO + 40 water box (configs.c2_mixture) is loaded into the COMMON blocks with the
intramolecular model of make_golden_shake.py (harmonic bonds, a seeded intramolecular reference
potential); each DMSO gets its two methyl groups as rotational groups of type ROT (axis S -> C,
the three H rotated), as the reference's own 200DMSO400Water.ato declares them, stepri > 0 and
a starting internrot.  After the cell list and pair store are built with the reference's
routines, molfit runs two whole-molecule cycles (nisum < intra) with rotfreq 1, so every DMSO
is first rotated internally and then moved whole.  Every cosf value molfit draws is recorded
in order (rotati's and rotatm's), so the device and the oracle can reproduce the chain bit for
bit.  tests/golden/rot.npz receives the inputs, the groups (0-based), and after each cycle the
coordinates, the store energies, the step arrays, ninter/nwhole/nmovem, fadds/faddbs and the
ran1 state.

The same box also runs two intramolecular cycles (nisum >= intra, molfit.py:124-267): every
molecule's atoms moved at random and tested on its intramolecular energy, then its methyl
groups rotated and tested on the intramolecular and intermolecular change, molecules in index
order; stepmi > 0 and a starting interntrans as make_golden_shake.py.  tests/golden/shake_rot.npz
receives the same fields plus nmovei per cycle.

With dihedral angles (dih_rot.npz, dih_shake.npz) the methyl groups are of type DIH, each with
one dihedral angle (base atoms S and C, orientation atoms O and the group's first H; 1.0 and 2.5
rad for the two methyls), dihtemp (tempdihreq) 1: en_mole_intra then adds tempdih * simt * en_mole_dihedral
(molfit.py:1345-1348, :1353) and en_atom_intra leaves the O-H pairs out of the reference potential
(:999-1020).  The cosines en_dihedral takes of the dihedral angles are not part of the recorded
draw cosines; their cosf/sinf values are written as dih_cos/dih_sin.
"""

from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)
sys.path.insert(0, HERE)

from epsr_python_translation_b200 import configs  # noqa: E402
import refstate  # noqa: E402
from make_golden import system_arrays  # noqa: E402

f32 = np.float32
REF = refstate.reference_root()


def run(s, out, seed=21, cycles=2, internrot=0.08, shake=False, interntrans_A=0.05, dih=False):
    from epsr26.common import clustercom, epsr16, molecom, molecom_mod, potential_par
    from epsr26.fortran import f32 as F, r4
    from epsr26.fortran.arrays import int_array
    from epsr26.library import ato_manipulation_rev4, cellneighbourlist, minimagec, molfit
    rng = np.random.default_rng(seed)
    nmt = s.nmoltype
    refstate.populate(s, rejrate=0.75, wholerot=[0.0556] * nmt, wholetrans=[f32(0.5) / s.dmax] * nmt)
    for k, v in system_arrays(s).items():
        out[k] = v
    # the intramolecular model (as make_golden_shake.py)
    molecom.tempangreq = f32(2.0)
    molecom.tempangwt = f32(2.0)
    for t, lab in enumerate(s.type_labels):
        molecom.amassa[t + 1] = f32(configs.TYPE_PARAMS[lab][3])
    npt = s.grid["npt"]
    xav = (rng.standard_normal((npt + 1, s.npairs)) * 0.3).astype(f32)
    xav1 = (rng.standard_normal((npt + 1, s.npairs)) * 3.0).astype(f32)
    potential_par.xav[: npt + 1, 1: s.npairs + 1] = xav
    potential_par.xav1[: npt + 1, 1: s.npairs + 1] = xav1
    maxbond = int(np.max(molecom.nbond[1: s.natom + 1]))
    out["nbond"] = np.array(molecom.nbond[1: s.natom + 1], np.int32)
    out["iabond"] = np.array(molecom.iabond[1: s.natom + 1, 1: maxbond + 1], np.int32) - 1
    out["tbond"] = np.array(molecom.tbond[1: s.natom + 1, 1: maxbond + 1], f32)
    out["amassa"] = np.array(molecom.amassa[1: s.ntype + 1], f32)
    out["amassr"] = np.array(molecom.amassr[1: s.npairs + 1], f32)
    out["xav"] = xav.T.copy()
    out["xav1"] = xav1.T.copy()
    # rotational groups: per DMSO (template atoms S 0, OD 1, C 2, C 3, H 4-9) the two methyls
    dmso = [m for m in range(s.nmol) if s.mtype[m] == 0]
    ng = 2 * len(dmso)
    molecom_mod.ngrrot = ng
    molecom_mod.rotgrp = np.array(["   "] + ["DIH" if dih else "ROT"] * ng, dtype=object)
    molecom_mod.labaxi = int_array(ng, 2)
    molecom_mod.nrot = int_array(ng)
    molecom_mod.rotf = int_array(ng)
    molecom_mod.rotl = int_array(ng)
    molecom_mod.mrot = int_array(ng)
    molecom_mod.nrottot = 3 * ng
    molecom_mod.labrot = int_array(3 * ng)
    axis, first, last, atoms = [], [], [], []
    nrf = np.zeros(s.nmol, np.int32)
    nrl = np.full(s.nmol, -1, np.int32)
    ngrot = np.zeros(s.nmol, np.int32)
    ig = 0
    ia = 0
    for m in dmso:
        a0 = int(s.naf[m])
        clustercom.ngrot[m + 1] = 2
        clustercom.nrf[m + 1] = ig + 1
        clustercom.nrl[m + 1] = ig + 2
        nrf[m], nrl[m], ngrot[m] = ig, ig + 1, 2
        for c, h0 in ((2, 4), (3, 7)):
            ig += 1
            molecom_mod.labaxi[ig, 1] = a0 + 0 + 1
            molecom_mod.labaxi[ig, 2] = a0 + c + 1
            molecom_mod.nrot[ig] = 3
            molecom_mod.mrot[ig] = m + 1
            molecom_mod.rotf[ig] = ia + 1
            axis.append((a0, a0 + c))
            first.append(ia)
            for k in range(3):
                ia += 1
                molecom_mod.labrot[ia] = a0 + h0 + k + 1
                atoms.append(a0 + h0 + k)
            molecom_mod.rotl[ig] = ia
            last.append(ia - 1)
    for m in range(s.nmol):
        for a in range(int(s.naf[m]), int(s.naf[m]) + int(s.nato[m])):
            molecom.mref[a + 1] = m + 1
    angles = (F(1.0), F(2.5))
    if dih:
        # one dihedral angle per methyl group: base atoms S, C; orientation atoms O (bonded to S)
        # and the group's first H (bonded to C)
        dih_atoms, dih_ang = [], []
        for ig in range(1, ng + 1):
            a_s, a_c = int(molecom_mod.labaxi[ig, 1]), int(molecom_mod.labaxi[ig, 2])
            a_h = int(molecom_mod.labrot[molecom_mod.rotf[ig]])
            a_o = a_s + 1
            molecom.ndihedralang[ig] = 1
            molecom.labrotdih[1, 1, ig] = a_o
            molecom.labrotdih[2, 1, ig] = a_h
            molecom.dihedralang[1, ig] = angles[(ig - 1) % 2]
            dih_atoms.append((a_o - 1, a_h - 1))
            dih_ang.append(angles[(ig - 1) % 2])
        molecom.tempdihreq = f32(1.0)    # fmolec1 and molfit set tempdihwt from it
        molecom.tempdihwt = molecom.tempdihreq
        molecom.tempdih = f32(f32(molecom.tempdihwt) * f32(molecom.tempb))
        out.update(dih_atoms=np.array(dih_atoms, np.int32), dih_grp0=np.arange(ng + 1, dtype=np.int32),
                   dih_isdih=np.ones(ng, np.int32), dih_cos=np.array([molfit.cosf(a) for a in dih_ang], f32),
                   dih_sin=np.array([molfit.sinf(a) for a in dih_ang], f32), tempdih=f32(molecom.tempdih))
    molecom.stepri = f32(1.0)
    ir0 = np.array([internrot] + [0.0] * (nmt - 1), f32)
    clustercom.internrot[1: nmt + 1] = ir0
    if shake:
        # the intramolecular moves: stepmi > 0, interntrans 0 for the first type (the trstepmin
        # start is taken) and interntrans_A for the others
        molecom.stepmi = f32(1.0)
        it0 = np.array([0.0] + [interntrans_A / float(s.dmax)] * (nmt - 1), f32)
        clustercom.interntrans[1: nmt + 1] = it0
        out["interntrans_in"] = it0
        out["stepmi"] = f32(molecom.stepmi)
    out.update(rot_axis=np.array(axis, np.int32), rot_first=np.array(first, np.int32),
               rot_last=np.array(last, np.int32), rot_atoms=np.array(atoms, np.int32), rot_nrf=nrf, rot_nrl=nrl,
               ngrot=ngrot, internrot_in=ir0,
               scal=np.array([epsr16.cellst / molecom.dmaxmol, molecom.sizefactor, molecom.tempb, molecom.tempangwt,
                              molecom.simt], f32))
    out["wholerot_in"] = np.array(clustercom.wholerot[1: nmt + 1], f32)
    out["wholetrans_in"] = np.array(clustercom.wholetrans[1: nmt + 1], f32)
    out["in_stepr"], out["in_stepm"] = f32(molecom.stepr), f32(molecom.stepm)
    out["in_rejrate"] = f32(epsr16.rejrate)
    out["in_natomr"] = np.int32(molecom.natomr)
    out["in_maxmolsize"] = f32(molecom.maxmolsize)
    sepmax = epsr16.xstar[epsr16.nptmax] + molecom.maxmolsize + r4(3.0) / clustercom.dmax
    out["in_sepmax"], out["in_nmolcell"] = f32(sepmax), np.int32(10)
    cellneighbourlist.initialise_cellneighbourlist(10, clustercom.xadd, clustercom.yadd, clustercom.zadd,
                                                   clustercom.nmol, sepmax)
    for im in range(1, s.nmol + 1):
        clustercom.xadd[im], clustercom.yadd[im], clustercom.zadd[im] = minimagec.minimagec(
            clustercom.xadd[im], clustercom.yadd[im], clustercom.zadd[im])
    molecom.tempang = molecom.tempangwt
    eintra = np.zeros(s.nmol, f32)
    for im in range(1, s.nmol + 1):
        e, _, _, _ = molfit.en_mole_intra(im, F(0), F(0), F(0))
        eintra[im - 1] = e
    out["eintra"] = eintra
    ato_manipulation_rev4.fmolec1(0, 0, F(0), F(0), F(0), F(0))
    for k, v in refstate.coords_state(s).items():
        out["in_" + k] = v
    for k, v in refstate.store_state().items():
        out["in_" + k] = v
    for k, v in refstate.ran1_state().items():
        out["ran1_before_" + k] = v
    rec = []
    orig_cosf = molfit.cosf

    def cosf_rec(x):
        v = orig_cosf(x)
        if not (dih and any(x == a for a in angles)):   # en_dihedral's fixed angles are not draws
            rec.append(v)
        return v

    molfit.cosf = cosf_rec
    fadds, faddbs, nisum = F(0.25), F(-0.5), 1
    out["fadds_in"], out["faddbs_in"] = fadds, faddbs
    try:
        for c in range(cycles):
            n0 = len(rec)
            if shake:
                fadds, faddbs, nisum = molfit.molfit(fadds, faddbs, 1, 1, 5, 0)
            else:
                fadds, faddbs, nisum = molfit.molfit(fadds, faddbs, nisum, 100, 1, 0)
            q = f"c{c}_"
            out[q + "cos"] = np.array(rec[n0:], f32)
            out[q + "fadds"], out[q + "faddbs"], out[q + "nisum"] = f32(fadds), f32(faddbs), np.int32(nisum)
            for k, v in refstate.coords_state(s).items():
                out[q + k] = v
            out[q + "ergpair"] = refstate.store_state()["ergpair"]
            for k in ("interntrans", "internrot", "wholerot", "wholetrans"):
                out[q + k] = np.array(getattr(clustercom, k)[1: nmt + 1], f32)
            for k in ("ninter", "nwhole", "nmovem", "nmovei"):
                out[q + k] = np.array(getattr(clustercom, k)[1:3, 1: nmt + 1], np.int32)
            out[q + "nstepreject"] = np.array(clustercom.nstepreject[1: s.nmol + 1], np.int32)
            for k, v in refstate.ran1_state().items():
                out[q + "ran1_after_" + k] = v
            print(f"cycle {c}: ninter {out[q + 'ninter'].tolist()} nmovei {out[q + 'nmovei'].tolist()} "
                  f"faddbs {faddbs} cos {len(rec) - n0}", flush=True)
    finally:
        molfit.cosf = orig_cosf
    out["cycles"] = np.int32(cycles)


if __name__ == "__main__":
    common, _ = refstate.load_reference(os.path.join(REF, "src"))
    out = {}
    which = sys.argv[1] if len(sys.argv) > 1 else "both"
    if which in ("both", "rot"):
        common.reset()
        run(configs.c2_mixture(seed=5, ndmso=20, nwater=40), out)
        path = os.path.join(HERE, "rot.npz")
        np.savez_compressed(path, **out)
        print("wrote", path)
    if which in ("dih",):
        for name, shake in (("dih_rot", False), ("dih_shake", True)):
            out = {}
            common.reset()
            run(configs.c2_mixture(seed=5, ndmso=20, nwater=40), out, seed=29, shake=shake, dih=True)
            path = os.path.join(HERE, name + ".npz")
            np.savez_compressed(path, **out)
            print("wrote", path)
    if which in ("both", "shake_rot"):
        out = {}
        common.reset()
        run(configs.c2_mixture(seed=5, ndmso=20, nwater=40), out, seed=23, shake=True)
        path = os.path.join(HERE, "shake_rot.npz")
        np.savez_compressed(path, **out)
        print("wrote", path)
