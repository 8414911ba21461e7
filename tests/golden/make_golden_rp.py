"""Golden vectors for the reference potential tables: generate_rp (epsr_standalone_rev3.py:5675-5873,
which calls generate_mp ato_manipulation_rev4.py:2816 first), made by running the reference
translation (epsr26) on seeded parameters.

Run in a container where the reference is importable (it is read-only; nothing is written
there):

    EPSR_REFERENCE=<reference checkout> PYTHONDONTWRITEBYTECODE=1 python tests/golden/make_golden_rp.py

Cases: "lj" (power 12, charged spheres of radii 0, 0.5 and 1.0 A so that every branch of chsph
is taken, the exponential repulsive core without a gradient limit), "gauss" (power 10, two
Gaussians per set of either sign, a harmonic repulsive core with a gradient limit,
coul_intra, refpotfac 0.8, pairs sharing coefficient sets) and "morse" (the modified Morse of
gauss6pot as the first added function, the exponential core with a gradient limit).
tests/golden/rp.npz receives the inputs and the six tables epot, epot1, ecoul, ecoul1, xav,
xav1 ([pair][j], j = 0..npt).
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

f32 = np.float32
REF = refstate.reference_root()
TABS = ("epot", "epot1", "ecoul", "ecoul1", "xav", "xav1")


def run_case(name, ep, out, *, ntype, power, seed, iref=None, ngauss=0, modmorse=False, harmonic=False,
             gradlimit=0.0, coul_intra=False, refpotfac=1.0, rmaxgr=14.0):
    from epsr26.common import clustercom, epsr16, epsrinput_par, molecom, potential_par as pp
    rng = np.random.default_rng(seed)
    g = configs.make_rgrid(0.03, rmaxgr, 9.0, 12.0)
    npt, npt2 = g["npt"], g["npt2"]
    dmax = f32(2.0 * rmaxgr)
    clustercom.dmax = dmax
    clustercom.nmol = 1
    epsr16.npt, epsr16.npt2, epsr16.npt1 = npt, npt2, g["npt1"]
    epsr16.x[: npt + 1] = g["x"]
    epsr16.xstar[: npt + 1] = (g["x"] / dmax).astype(f32)
    pairs = [(i, j) for i in range(ntype) for j in range(i, ntype)]
    npairs = len(pairs)
    iref = list(range(npairs)) if iref is None else list(iref)
    nsets = max(iref) + 1
    molecom.npairs, molecom.ntype, molecom.natom = npairs, ntype, 0
    molecom.power = f32(power)
    molecom.ecore, molecom.dcore, molecom.sizefactor = f32(0.5), f32(2.2), f32(1.0)
    molecom.coul_intra, molecom.coul_intra_fac = bool(coul_intra), f32(0.7)
    qradius = np.array([0.0, 0.5, 1.0, 0.3][:ntype], f32)
    molecom.qradius[1: ntype + 1] = qradius
    ecor = rng.uniform(0.1, 1.5, npairs).astype(f32)
    dcor = rng.uniform(2.5, 3.6, npairs).astype(f32)
    qcor = (rng.uniform(-1.0, 1.0, npairs) * 138.9).astype(f32)
    for p, (i, j) in enumerate(pairs):
        molecom.n1extr[p + 1], molecom.n2extr[p + 1] = i + 1, j + 1
        molecom.ecor[p + 1], molecom.dcor[p + 1], molecom.qcor[p + 1] = ecor[p], dcor[p], qcor[p]
        pp.irefpcof[p + 1] = iref[p] + 1
    coulfac = rng.uniform(0.8, 1.2, nsets).astype(f32)
    pcoefex = rng.uniform(0.5, 2.0, nsets).astype(f32)
    rminex = rng.uniform(1.5, 2.5, nsets).astype(f32)
    rminex[0] = 0.0                     # a set without a repulsive core
    maxg = max(ngauss, 1)
    wpg = rng.uniform(0.1, 0.4, (nsets, maxg)).astype(f32)
    rpg = rng.uniform(2.0, 5.0, (nsets, maxg)).astype(f32)
    hpg = (rng.uniform(0.2, 1.0, (nsets, maxg)) * rng.choice([-1.0, 1.0], (nsets, maxg))).astype(f32)
    npg = np.full(nsets, ngauss, np.int32)
    for k in range(nsets):
        pp.coulfac[k + 1], pp.pcoefex[k + 1], pp.rminex[k + 1], pp.rmaxex[k + 1] = coulfac[k], pcoefex[k], rminex[k], 0.0
        pp.npgauss[k + 1] = npg[k]
        for ig in range(maxg):
            pp.wpgauss[ig + 1, k + 1], pp.rpgauss[ig + 1, k + 1], pp.hpgauss[ig + 1, k + 1] = wpg[k, ig], rpg[k, ig], hpg[k, ig]
    pp.addpotential = "modmorse" if modmorse else ""
    pp.harmonic = bool(harmonic)
    pp.refpotfac = f32(refpotfac)
    wfac = configs.truncate_lj(g["x"].astype(np.float64), 9.0, 12.0).astype(f32)
    wfac[npt] = 0.0
    wfacc = configs.truncate_coul(np.maximum(g["x"].astype(np.float64), 1e-4), 12.0).astype(f32)
    wfacc[npt] = 0.0
    pp.wfac[: npt + 1], pp.wfacc[: npt + 1] = wfac, wfacc
    epsrinput_par.expecf, epsrinput_par.expecfpwr = f32(0.3), f32(gradlimit)
    p = name + "_"
    out.update({p + "x": g["x"], p + "xstar": (g["x"] / dmax).astype(f32), p + "wfac": wfac, p + "wfacc": wfacc,
                p + "dims": np.array([npairs, npt, npt2, ntype, nsets, maxg]),
                p + "scal": np.array([power, 0.5, 2.2, 1.0, refpotfac, 0.3, gradlimit, float(harmonic),
                                      float(modmorse), float(coul_intra), 0.7], f32),
                p + "pairs": np.array(pairs, np.int32), p + "iref": np.array(iref, np.int32), p + "qradius": qradius,
                p + "ecor": ecor, p + "dcor": dcor, p + "qcor": qcor, p + "coulfac": coulfac, p + "pcoefex": pcoefex,
                p + "rminex": rminex, p + "npgauss": npg, p + "wpgauss": wpg, p + "rpgauss": rpg, p + "hpgauss": hpg})
    ep.generate_rp()
    for k in TABS:
        out[p + k] = np.array(getattr(pp, k)[: npt + 1, 1: npairs + 1], f32).T.copy()
    print(f"[{name}] npairs {npairs} npt {npt} done", flush=True)


if __name__ == "__main__":
    common, _ = refstate.load_reference(os.path.join(REF, "src"))
    import importlib
    ep = importlib.import_module("epsr26.programs.epsr_standalone_rev3")
    out = {}
    common.reset()
    run_case("lj", ep, out, ntype=3, power=12.0, seed=1)
    common.reset()
    run_case("gauss", ep, out, ntype=3, power=10.0, seed=2, iref=[0, 1, 2, 1, 0, 3], ngauss=2, harmonic=True,
             gradlimit=5.0, coul_intra=True, refpotfac=0.8)
    common.reset()
    run_case("morse", ep, out, ntype=2, power=12.0, seed=3, ngauss=2, modmorse=True, gradlimit=3.0)
    path = os.path.join(HERE, "rp.npz")
    np.savez_compressed(path, **out)
    print("wrote", path)
