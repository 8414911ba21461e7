"""Golden vectors for generate_ep (epsr_standalone_rev3.py:5876-): the empirical-potential
tables rebuilt from the EP coefficients, made by running the reference translation (epsr26)
on seeded state.

Run in a container where the reference is importable (it is read-only; nothing is written
there):

    EPSR_REFERENCE=<reference checkout> PYTHONDONTWRITEBYTECODE=1 python tests/golden/make_golden_ep.py

Each case fills potential_par (Poisson basis of the reference's own default size for
rminpt 9 / rmaxpt 12 A: pdstep 0.1, pdmin 1 + pdstep/rminpt, 116 terms), the r grid of
configs.make_rgrid, seeded coefficients pcoefp, a seeded truncation wfac, seeded Coulomb
tables and seeded previous EP tables (generate_ep reads a few entries it does not rewrite),
and calls generate_ep two or three times in a row.  The cases cover every pressfac rule
(the erequnit floor, the cap at 1 without ereqstep, a shrink, no absolute energy) and a
coefficient set shared by two pairs (multiply_pot_coeffs scales it once per pair).  tests/golden/ep.npz receives the inputs, the basis
matrix expgr the reference built (calc_pwrexpr_grad), and the state after each call
(0-based copies of the 1-based arrays: [j, pair] for tables, [ic, pair] for coefficients).
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


def run_case(name, ep, npairs, rmaxgr, absolute_energy, erequnit, ereqstep, seed, out, ncalls=2, iref=None,
             gaussian=False, psigma2=0.004, rbroad=0.0):
    from epsr26.common import clustercom, epsr16, epsrinput_par, molecom, potential_par as pp
    from epsr26.fortran import r4
    rng = np.random.default_rng(seed)
    g = configs.make_rgrid(0.03, rmaxgr, 9.0, 12.0)
    npt, npt2 = g["npt"], g["npt2"]
    dmax = f32(2.0 * rmaxgr)
    clustercom.dmax = dmax
    epsr16.npt, epsr16.npt2, epsr16.npt1 = npt, npt2, g["npt1"]
    epsr16.x[: npt + 1] = g["x"]
    epsr16.xstar[: npt + 1] = (g["x"] / dmax).astype(f32)
    epsr16.rho = f32(0.1)
    molecom.npairs = npairs
    epsrinput_par.rminpt, epsrinput_par.rmaxpt, epsrinput_par.rbroad = f32(9.0), f32(12.0), f32(rbroad)
    pp.pdstep = r4(0.1)
    pp.pdmin = r4(1.0) + pp.pdstep / epsrinput_par.rminpt
    pp.pdmax = epsrinput_par.rmaxpt
    pp.ncoeffp = nterms = 116
    pp.psigma2 = r4(psigma2)
    pp.gaussian = bool(gaussian)
    iref = list(range(1, npairs + 1)) if iref is None else list(iref)   # 1-based set of each pair
    nsets = max(iref)
    pp.npairspcof = nsets
    for ip in range(1, npairs + 1):
        pp.irefpcof[ip] = iref[ip - 1]
    for k in range(1, nsets + 1):
        pp.npgauss[k] = 0
    pc = np.zeros((nterms + 1, nsets), f32)
    pc[1] = rng.uniform(0.5, 1.5, nsets).astype(f32)           # amplitude of each set's EP
    pc[2:] = (rng.standard_normal((nterms - 1, nsets)) * 0.05).astype(f32)
    pp.pcoefp[1: nterms + 1, 1: nsets + 1] = pc[1:]
    wfac = np.ones(npt + 1, f32)
    r = g["x"]
    taper = (r > 9.0) & (r < 12.0)
    wfac[taper] = (0.5 * (1.0 + np.cos(np.pi * (r[taper] - 9.0) / 3.0))).astype(f32)
    wfac[r >= 12.0] = f32(0.0)
    pp.wfac[: npt + 1] = wfac
    tabs = {}
    for k in ("ecoul", "xavs", "xavs1", "xavtot", "xavtot1"):
        v = (rng.standard_normal((npt + 1, npairs)) * 0.2).astype(f32)
        getattr(pp, k)[: npt + 1, 1: npairs + 1] = v
        tabs[k] = v
    pp.absolute_energy, pp.erequnit, pp.ereqstep = f32(absolute_energy), f32(erequnit), f32(ereqstep)
    pp.potfac, pp.potfacamp = f32(0.2), f32(0.5)
    for k, v in tabs.items():
        out[f"{name}_in_{k}"] = v
    out[f"{name}_in_pcoefp"] = pc
    out[f"{name}_wfac"] = wfac
    out[f"{name}_x"] = g["x"]
    out[f"{name}_xstar"] = (g["x"] / dmax).astype(f32)
    out[f"{name}_dims"] = np.array([npairs, npt, npt2, nterms, ncalls])
    out[f"{name}_iref"] = np.array(iref, np.int32) - 1
    out[f"{name}_scal"] = np.array([dmax, absolute_energy, erequnit, ereqstep, 0.2, 0.5], f32)
    # the basis parameters: gaussian, pdmin, pdstep, pdmax, psigma2, rho, rbroad
    out[f"{name}_basis"] = np.array([float(gaussian), pp.pdmin, pp.pdstep, pp.pdmax, pp.psigma2, epsr16.rho,
                                     epsrinput_par.rbroad], f32)
    for c in range(ncalls):
        ep.generate_ep(True)
        if c == 0:
            out[f"{name}_expgr"] = np.array(pp.expgr[1: npt2 * nterms + 1], f32)
        for k in ("xavs", "xavs1", "xavtot", "xavtot1"):
            out[f"{name}_c{c}_{k}"] = np.array(getattr(pp, k)[: npt + 1, 1: npairs + 1], f32)
        out[f"{name}_c{c}_pcoefp"] = np.array(pp.pcoefp[: nterms + 1, 1: nsets + 1], f32)
        out[f"{name}_c{c}_pwtold"] = np.array(pp.pwtold[: nterms + 1], f32)
        out[f"{name}_c{c}_potfac"] = np.float32(pp.potfac)
    print(f"[{name}] npt {npt} npt2 {npt2} done", flush=True)


if __name__ == "__main__":
    common, ep_prog = refstate.load_reference(os.path.join(REF, "src"))
    import importlib
    ep = importlib.import_module("epsr26.programs.epsr_standalone_rev3")
    out = {}
    common.reset()
    run_case("small", ep, npairs=3, rmaxgr=15.0, absolute_energy=3.0, erequnit=0.5, ereqstep=0.0, seed=1, out=out)
    common.reset()
    run_case("noabs", ep, npairs=4, rmaxgr=13.0, absolute_energy=0.0, erequnit=0.0, ereqstep=0.0, seed=2, out=out)
    common.reset()
    run_case("unit", ep, npairs=2, rmaxgr=14.0, absolute_energy=0.2, erequnit=20.0, ereqstep=1.0, seed=3, out=out)
    common.reset()
    run_case("cap", ep, npairs=3, rmaxgr=15.0, absolute_energy=3.0, erequnit=0.1, ereqstep=0.0, seed=4, out=out)
    common.reset()
    run_case("shrink", ep, npairs=2, rmaxgr=16.0, absolute_energy=0.1, erequnit=0.05, ereqstep=0.0, seed=5, out=out,
             ncalls=3)
    common.reset()
    run_case("shared", ep, npairs=3, rmaxgr=15.0, absolute_energy=3.0, erequnit=0.5, ereqstep=0.0, seed=6, out=out,
             iref=[1, 2, 1], rbroad=0.02)
    common.reset()
    run_case("gauss", ep, npairs=3, rmaxgr=14.0, absolute_energy=1.0, erequnit=0.2, ereqstep=0.0, seed=7, out=out,
             gaussian=True, psigma2=0.1, rbroad=0.02)
    path = os.path.join(HERE, "ep.npz")
    np.savez_compressed(path, **out)
    print("wrote", path)
