"""Golden vectors for the intramolecular branch of molfit (molfit.py:124-174, taken when
nisum >= intra) and en_mole_intra (:1327), made by running the reference translation (epsr26)
on seeded systems.

Run in a container where the reference is importable (it is read-only; nothing is written
there):

    EPSR_REFERENCE=<reference checkout> PYTHONDONTWRITEBYTECODE=1 python tests/golden/make_golden_shake.py

Each case loads a configs system into the COMMON blocks (refstate.populate: harmonic bonds
from the molecule templates, water's H-H pair as a bond-angle pair), then sets what this branch
reads beyond the whole-molecule path: stepmi > 0, the atom masses amassa, a seeded
intramolecular reference potential xav/xav1, tempangreq 2 (fmolec1 copies it to tempangwt,
which molfit uses, so bond-angle pairs are weighted),
and per type interntrans (0 for the first type, so the trstepmin start is taken).  It builds the
cell list and the pair store with the reference's own routines and runs two molfit cycles with
nisum = intra = 1.  tests/golden/shake.npz receives, per case, the inputs, the intramolecular
energies before the cycles, and after each cycle the coordinates, the store energies, the step
arrays, nmovei, fadds/faddbs and the ran1 state.
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


def run_case(name, s, out, *, refine_intra=False, seed=0, cycles=2, interntrans_A=0.05):
    from epsr26.common import clustercom, epsr16, molecom, potential_par
    from epsr26.common import ergpairreference as erd
    from epsr26.fortran import f32 as F, r4
    from epsr26.library import ato_manipulation_rev4, cellneighbourlist, minimagec, molfit
    rng = np.random.default_rng(seed)
    nmt = s.nmoltype
    refstate.populate(s, rejrate=0.75, wholerot=[0.0556] * nmt, wholetrans=[f32(0.5) / s.dmax] * nmt)
    p = name + "_"
    for k, v in system_arrays(s).items():
        out[p + k] = v
    # what the intramolecular branch reads beyond the whole-molecule path
    molecom.stepmi = f32(1.0)
    molecom.tempangreq = f32(2.0)      # fmolec1 sets tempangwt = tempangreq (ato_manipulation_rev4.py:2425)
    molecom.tempangwt = f32(2.0)
    molecom.refine_intra = bool(refine_intra)
    molecom.refine_intra_fac = f32(0.5)
    for t, lab in enumerate(s.type_labels):
        molecom.amassa[t + 1] = f32(configs.TYPE_PARAMS[lab][3])
    npt = s.grid["npt"]
    xav = (rng.standard_normal((npt + 1, s.npairs)) * 0.3).astype(f32)
    xav1 = (rng.standard_normal((npt + 1, s.npairs)) * 3.0).astype(f32)
    potential_par.xav[: npt + 1, 1: s.npairs + 1] = xav
    potential_par.xav1[: npt + 1, 1: s.npairs + 1] = xav1
    it0 = np.array([0.0] + [interntrans_A / float(s.dmax)] * (nmt - 1), f32)
    clustercom.interntrans[1: nmt + 1] = it0
    clustercom.internrot[1: nmt + 1] = f32(0.01)
    maxbond = int(np.max(molecom.nbond[1: s.natom + 1]))
    out[p + "nbond"] = np.array(molecom.nbond[1: s.natom + 1], np.int32)
    out[p + "iabond"] = np.array(molecom.iabond[1: s.natom + 1, 1: maxbond + 1], np.int32) - 1
    out[p + "tbond"] = np.array(molecom.tbond[1: s.natom + 1, 1: maxbond + 1], f32)
    out[p + "amassa"] = np.array(molecom.amassa[1: s.ntype + 1], f32)
    out[p + "amassr"] = np.array(molecom.amassr[1: s.npairs + 1], f32)
    out[p + "xav"] = xav.T.copy()
    out[p + "xav1"] = xav1.T.copy()
    out[p + "scal"] = np.array([epsr16.cellst / molecom.dmaxmol, molecom.sizefactor, molecom.tempb,
                                molecom.tempangwt, molecom.simt, float(refine_intra), molecom.refine_intra_fac,
                                molecom.stepmi], f32)
    out[p + "interntrans_in"] = it0
    out[p + "internrot_in"] = np.array(clustercom.internrot[1: nmt + 1], f32)
    out[p + "wholerot_in"] = np.array(clustercom.wholerot[1: nmt + 1], f32)
    out[p + "wholetrans_in"] = np.array(clustercom.wholetrans[1: nmt + 1], f32)
    # the keys the drop-in tests' COMMON stand-ins read (tests/fake_common.py)
    out[p + "in_wholerot"], out[p + "in_wholetrans"] = out[p + "wholerot_in"], out[p + "wholetrans_in"]
    out[p + "in_stepr"], out[p + "in_stepm"] = f32(molecom.stepr), f32(molecom.stepm)
    out[p + "in_rejrate"] = f32(epsr16.rejrate)
    out[p + "in_natomr"] = np.int32(molecom.natomr)
    out[p + "in_maxmolsize"] = f32(molecom.maxmolsize)
    # cell list, intramolecular energies and the pair store, as the reference loop builds them
    sepmax = epsr16.xstar[epsr16.nptmax] + molecom.maxmolsize + r4(3.0) / clustercom.dmax
    out[p + "in_sepmax"], out[p + "in_nmolcell"] = f32(sepmax), np.int32(10)
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
    out[p + "eintra"] = eintra
    ato_manipulation_rev4.fmolec1(0, 0, F(0), F(0), F(0), F(0))
    for k, v in refstate.coords_state(s).items():
        out[p + "in_" + k] = v
    for k, v in refstate.store_state().items():
        out[p + "in_" + k] = v
    for k, v in refstate.ran1_state().items():
        out[p + "ran1_before_" + k] = v
    ergold = getattr(erd, "ergold", None)
    out[p + "ergold1_in"] = f32(ergold[1] if ergold is not None and ergold.shape[0] > 1 else 0.0)
    fadds, faddbs, nisum = F(0.25), F(-0.5), 1
    out[p + "fadds_in"], out[p + "faddbs_in"] = fadds, faddbs
    for c in range(cycles):
        fadds, faddbs, nisum = molfit.molfit(fadds, faddbs, nisum, 1, 5, 0)
        q = f"{p}c{c}_"
        out[q + "fadds"], out[q + "faddbs"], out[q + "nisum"] = f32(fadds), f32(faddbs), np.int32(nisum)
        for k, v in refstate.coords_state(s).items():
            out[q + k] = v
        st = refstate.store_state()
        out[q + "ergpair"] = st["ergpair"]
        for k in ("interntrans", "internrot", "wholerot", "wholetrans"):
            out[q + k] = np.array(getattr(clustercom, k)[1: nmt + 1], f32)
        for k in ("nmovei", "nwhole", "nmovem"):
            out[q + k] = np.array(getattr(clustercom, k)[1:3, 1: nmt + 1], np.int32)
        for k, v in refstate.ran1_state().items():
            out[q + "ran1_after_" + k] = v
        acc = out[q + "nmovei"]
        print(f"[{name}] cycle {c}: tries {acc[0].tolist()} rejected {acc[1].tolist()} faddbs {faddbs}", flush=True)
    out[p + "cycles"] = np.int32(cycles)


if __name__ == "__main__":
    common, _ = refstate.load_reference(os.path.join(REF, "src"))
    out = {}
    common.reset()
    run_case("mix", configs.c2_mixture(seed=5, ndmso=20, nwater=40), out, seed=11)
    common.reset()
    run_case("water", configs.c1_water(seed=6), out, refine_intra=True, seed=12, interntrans_A=0.02)
    path = os.path.join(HERE, "shake.npz")
    np.savez_compressed(path, **out)
    print("wrote", path)
