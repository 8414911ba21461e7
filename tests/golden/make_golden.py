"""Generate golden vectors by running the reference translation (epsr26) on seeded systems.

Run in a container where the reference is importable (it is read-only; nothing is written
there):

    EPSR_REFERENCE=<reference checkout> PYTHONDONTWRITEBYTECODE=1 python tests/golden/make_golden.py [case ...]

Each case writes ``tests/golden/<case>.npz`` with the system inputs and, per routine, the
reference's outputs:

* ``initialise_cellneighbourlist`` (cellneighbourlist.py:23) cell arrays;
* ``fmolec1`` (ato_manipulation_rev4.py:2374) pair-energy store + ftest/ftestb, with the
  per-molecule intramolecular energies from ``en_mole_intra`` (molfit.py:1327);
* ``molfit`` whole-molecule cycles (molfit.py:52): per-move ``en_change`` value, the
  three ``cosf`` values of ``rotatm`` and the ran1 draws, then coordinates, store,
  counters and step sizes after each cycle;
* ``atogen`` (ato_manipulation_rev4.py:3640): normalised ``wav``, ``potex``;
* ``gensq`` (epsr_standalone_rev3.py:4731) and ``stog`` (ato_manipulation_rev4.py:4067);
* ``fit_expansion`` (epsr_standalone_rev3.py:4806) on a synthetic basis;
* ``ran1`` (auxiliary_routines.py:324) streams; the gfortran bit patterns of the
  reference's own ``tests/library/data/ran1_reference.txt`` are converted to
  ``ran1_reference.npz``.
"""

from __future__ import annotations

import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)
sys.path.insert(0, HERE)

from epsr_python_translation_b200 import configs  # noqa: E402
import refstate  # noqa: E402

f32 = np.float32
REF = refstate.reference_root()


def system_arrays(s):
    g = s.grid
    return dict(
        sys_L=np.float64(s.L), sys_dmax=np.float32(s.dmax), sys_itype=s.itype, sys_mtype=s.mtype, sys_naf=s.naf,
        sys_nato=s.nato, sys_xa=s.xa, sys_ya=s.ya, sys_za=s.za, sys_xadd=s.xadd, sys_yadd=s.yadd, sys_zadd=s.zadd,
        sys_npairref=s.npairref, sys_n1extr=s.n1extr, sys_n2extr=s.n2extr, sys_cellst=np.float32(s.cellst),
        sys_x=g["x"], sys_npt=np.int32(g["npt"]), sys_npt1=np.int32(g["npt1"]), sys_npt2=np.int32(g["npt2"]),
        sys_nptmin=np.int32(g["nptmin"]), sys_nptmax=np.int32(g["nptmax"]), sys_xstar=s.xstar,
        sys_xavs=s.xavs, sys_xavs1=s.xavs1, sys_ecoul=s.ecoul, sys_ecoul1=s.ecoul1,
        sys_simt=np.float32(s.simt), sys_temperature=np.float64(s.temperature), sys_nmoltype=np.int32(s.nmoltype),
        sys_cfrac=s.cfrac, sys_ntype=np.int32(s.ntype))


def run_case(name, s, *, cycles=2, ngrsamples=0, nq=600, qstep=0.05, transforms=True, wholerot=0.0556,
             wholetrans_A=0.5, rejrate=0.75, nmolcell=10):
    from epsr26.common import cellneighbourlist as cnl
    from epsr26.common import clustercom, epsr16, molecom, potential_par
    from epsr26.common import epsr_dimension
    from epsr26.fortran import f32 as F, r4
    from epsr26.library import (ato_manipulation_rev4, auxiliary_routines, cellneighbourlist, minimagec, molfit)
    from epsr26.fortran.arrays import real_array
    ep = sys.modules["epsr26.programs.epsr_standalone_rev3"]

    t0 = time.time()
    nmt = s.nmoltype
    refstate.populate(s, rejrate=rejrate, wholerot=[wholerot] * nmt,
                      wholetrans=[f32(wholetrans_A) / s.dmax] * nmt)
    out = system_arrays(s)
    out["in_wholerot"] = np.array(clustercom.wholerot[1:nmt + 1])
    out["in_wholetrans"] = np.array(clustercom.wholetrans[1:nmt + 1])
    out["in_rejrate"] = np.float32(rejrate)
    out["in_stepr"] = np.float32(molecom.stepr)
    out["in_stepm"] = np.float32(molecom.stepm)
    out["in_natomr"] = np.int32(molecom.natomr)
    out["in_maxmolsize"] = np.float32(molecom.maxmolsize)
    # --- cell list (runepsr17 epsr_standalone_rev3.py:1259-1266)
    sepmax = epsr16.xstar[epsr16.nptmax] + molecom.maxmolsize + r4(3.0) / clustercom.dmax
    out["in_sepmax"] = np.float32(sepmax)
    out["in_nmolcell"] = np.int32(nmolcell)
    cellneighbourlist.initialise_cellneighbourlist(nmolcell, clustercom.xadd, clustercom.yadd, clustercom.zadd,
                                                   clustercom.nmol, sepmax)
    for k, v in refstate.cell_state(s.nmol).items():
        out["cell_" + k] = v
    for im in range(1, s.nmol + 1):
        clustercom.xadd[im], clustercom.yadd[im], clustercom.zadd[im] = minimagec.minimagec(
            clustercom.xadd[im], clustercom.yadd[im], clustercom.zadd[im])
    # --- intramolecular energies (the slot-1 input of fmolec1)
    eintra = np.zeros(s.nmol, dtype=f32)
    for im in range(1, s.nmol + 1):
        e, _, _, _ = molfit.en_mole_intra(im, F(0), F(0), F(0))
        eintra[im - 1] = e
    out["in_eintra"] = eintra
    # --- fmolec1
    ierr, nth, ftest, ftestb, fteth, fcc = ato_manipulation_rev4.fmolec1(0, 0, F(0), F(0), F(0), F(0))
    out["fm_ftest"] = np.float32(ftest)
    out["fm_ftestb"] = np.float32(ftestb)
    for k, v in refstate.store_state().items():
        out["fm_" + k] = v
    print(f"[{name}] fmolec1 done {time.time() - t0:.1f}s nnbrefmax={out['fm_nnbrefmax']} "
          f"nergpair={out['fm_nergpair']}", flush=True)
    # --- molfit cycles, instrumented through module attributes (the reference's trace mechanism)
    rec = {"ran1": [], "cos": [], "den": [], "im": []}
    orig_ran1 = auxiliary_routines.ran1
    orig_cosf = molfit.cosf
    orig_en_change = molfit.en_change

    def ran1_rec():
        v = orig_ran1()
        rec["ran1"].append(v)
        return v

    def cosf_rec(x):
        v = orig_cosf(x)
        rec["cos"].append(v)
        return v

    def en_change_rec(im):
        v = orig_en_change(im)
        rec["den"].append(v)
        rec["im"].append(im)
        return v

    for k, v in refstate.ran1_state().items():
        out["mf_ran1_before_" + k] = v
    auxiliary_routines.ran1 = ran1_rec
    molfit.cosf = cosf_rec
    molfit.en_change = en_change_rec
    fadds = F(0)
    faddbs = F(0)
    nisum = 1
    try:
        for c in range(cycles):
            nd0, nc0, ne0 = len(rec["ran1"]), len(rec["cos"]), len(rec["den"])
            fadds, faddbs, nisum = molfit.molfit(fadds, faddbs, nisum, 100, 5, 0)
            p = f"mf{c}_"
            out[p + "fadds"] = np.float32(fadds)
            out[p + "nisum"] = np.int32(nisum)
            out[p + "ran1"] = np.array(rec["ran1"][nd0:], dtype=np.float32)
            out[p + "cos"] = np.array(rec["cos"][nc0:], dtype=np.float32)
            out[p + "den"] = np.array(rec["den"][ne0:], dtype=np.float32)
            out[p + "im"] = np.array(rec["im"][ne0:], dtype=np.int32)
            for k, v in refstate.coords_state(s).items():
                out[p + k] = v
            for k, v in refstate.store_state().items():
                out[p + k] = v
            out[p + "wholerot"] = np.array(clustercom.wholerot[1:nmt + 1])
            out[p + "wholetrans"] = np.array(clustercom.wholetrans[1:nmt + 1])
            out[p + "nwhole"] = np.array(clustercom.nwhole[1:3, 1:nmt + 1], dtype=np.int32)
            out[p + "nmovem"] = np.array(clustercom.nmovem[1:3, 1:nmt + 1], dtype=np.int32)
            out[p + "nstepreject"] = np.array(clustercom.nstepreject[1:s.nmol + 1], dtype=np.int32)
            for k, v in refstate.ran1_state().items():
                out[p + "ran1_after_" + k] = v
            print(f"[{name}] molfit cycle {c} done {time.time() - t0:.1f}s moves={len(rec['den']) - ne0}",
                  flush=True)
    finally:
        auxiliary_routines.ran1 = orig_ran1
        molfit.cosf = orig_cosf
        molfit.en_change = orig_en_change
    out["mf_cycles"] = np.int32(cycles)
    # --- atogen
    for k, v in refstate.ran1_state().items():
        out["ag_ran1_before_" + k] = v
    mpz, mpairs = epsr_dimension.mpz, epsr_dimension.mpairs
    wav = real_array(2, mpz, mpairs)
    ngr = ato_manipulation_rev4.atogen(wav, ngrsamples)
    npt1 = epsr16.npt1
    out["ag_ngrsamples_in"] = np.int32(ngrsamples)
    out["ag_ngrsamples"] = np.int32(ngr)
    out["ag_wav"] = np.array(wav[1:3, 1:npt1 + 1, 1:s.npairs + 1], dtype=np.float32)
    out["ag_potex"] = np.array(potential_par.potex[1:s.npairs + 1], dtype=np.float32)
    out["ag_rminex"] = np.array(potential_par.rminex[1:s.npairs + 1], dtype=np.float32)
    for k, v in refstate.ran1_state().items():
        out["ag_ran1_after_" + k] = v
    print(f"[{name}] atogen done {time.time() - t0:.1f}s", flush=True)
    if transforms:
        # --- gensq with a foqols-like table
        q = configs.qgrid(nq, qstep)
        F_, ycoh = configs.transform_table(s, q, npt1)
        epsr16.foqols[: npt1 + 1, : nq + 1] = F_
        epsr16.ycoh[: ycoh.shape[0]] = ycoh
        qfull = real_array(epsr_dimension.mpts)
        qfull[: nq + 1] = q
        sofq = real_array(2, epsr_dimension.mpts, mpairs)
        ep.gensq(nq, qfull, sofq, wav)
        out["gs_nq"] = np.int32(nq)
        out["gs_q"] = q
        out["gs_foqols"] = F_
        out["gs_ycoh"] = ycoh
        out["gs_sofq"] = np.array(sofq[1:3, 1:nq + 1, 1:s.npairs + 1], dtype=np.float32)
        print(f"[{name}] gensq done {time.time() - t0:.1f}s", flush=True)
        # --- stog of the intermolecular S(Q) back to r
        nr = npt1
        sq2 = real_array(nq, s.npairs)
        sq2[1:nq + 1, 1:s.npairs + 1] = sofq[2, 1:nq + 1, 1:s.npairs + 1]
        r = real_array(nr)
        r[1:nr + 1] = epsr16.x[1:nr + 1]
        gofr = real_array(nr, s.npairs)
        nqmin = np.zeros(s.npairs + 1, dtype=np.int32)
        nqmax = np.zeros(s.npairs + 1, dtype=np.int32)
        nqmin[1:] = 2
        nqmax[1:] = nq
        xwt = real_array(s.npairs)
        xwt[1:] = np.linspace(0.5, 1.5, s.npairs).astype(f32)
        rho = F(s.natom) / F(s.L ** 3)
        ato_manipulation_rev4.stog(rho, qfull, sq2, r, gofr, nqmin, nqmax, nr, s.npairs, nq, nr, s.npairs, xwt)
        out["sg_rho"] = np.float32(rho)
        out["sg_r"] = np.array(r[1:nr + 1])
        out["sg_xwt"] = np.array(xwt[1:])
        out["sg_nqmin"] = nqmin[1:]
        out["sg_nqmax"] = nqmax[1:]
        out["sg_gofr"] = np.array(gofr[1:nr + 1, 1:], dtype=np.float32)
        print(f"[{name}] stog done {time.time() - t0:.1f}s", flush=True)
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
    print(f"[{name}] wrote {name}.npz in {time.time() - t0:.1f}s", flush=True)


def run_fit(name="fitexp", nq=160, nterms=40, seed=5, nfreq=10, stepr=0.01):
    from epsr26.fortran import f32 as F, r4
    from epsr26.fortran.arrays import real_array
    from epsr26.common import ran1com
    ep = sys.modules["epsr26.programs.epsr_standalone_rev3"]
    from epsr26 import common
    common.reset()
    prob = configs.fit_problem(nq=nq, nterms=nterms, seed=seed)
    out = dict(fx_yin=prob["yin"], fx_expr=prob["expr"], fx_nterms=np.int32(nterms), fx_npt=np.int32(nq),
               fx_nfreq=np.int32(nfreq), fx_stepr_in=np.float32(stepr))
    # advance the stream a little so the fit does not start at the initial state
    from epsr26.library import auxiliary_routines
    for _ in range(37):
        auxiliary_routines.ran1()
    for k, v in refstate.ran1_state().items():
        out["fx_ran1_before_" + k] = v
    runs = [dict(ncfirst=1, acceptr=r4(0.0005), wt0=0.0), dict(ncfirst=3, acceptr=r4(0.002), wt0=0.02)]
    for k, run in enumerate(runs):
        wt = real_array(nterms)
        wtold = real_array(nterms)
        rng = np.random.default_rng(seed + k)
        wtold[1:] = (run["wt0"] * rng.uniform(-1, 1, nterms)).astype(f32)
        if k == 1:
            wtold[5] = f32(1.5)     # exercise the |wtold| >= 1 multiplicative branch
        yout = real_array(nq)
        p = f"fx{k}_"
        out[p + "wtold_in"] = np.array(wtold[1:])
        out[p + "ncfirst"] = np.int32(run["ncfirst"])
        out[p + "acceptr_in"] = np.float32(run["acceptr"])
        for kk, v in refstate.ran1_state().items():
            out[p + "ran1_before_" + kk] = v
        t0 = time.time()
        res = ep.fit_expansion(prob["yin"], prob["expr"], yout, wt, wtold, F(stepr), run["acceptr"], F(0), F(0),
                               1, nq, run["ncfirst"], nterms, 1000, nfreq)
        stepr_o, acceptr_o, rejrat_o, chisq_o = res
        out[p + "stepr"] = np.float32(stepr_o)
        out[p + "acceptr"] = np.float32(acceptr_o)
        out[p + "rejrat"] = np.float32(rejrat_o)
        out[p + "chisq"] = np.float32(chisq_o)
        out[p + "wt"] = np.array(wt[1:])
        out[p + "wtold"] = np.array(wtold[1:])
        out[p + "yout"] = np.array(yout[1:])
        for kk, v in refstate.ran1_state().items():
            out[p + "ran1_after_" + kk] = v
        print(f"[{name}] fit {k} done in {time.time() - t0:.1f}s mcall={ran1com.mcall}", flush=True)
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)


def run_ran1(name="ran1_stream"):
    """ran1 from the epsr start state (idum=0 -> initialised with idum=1) and seeded starts,
    plus the reference's committed gfortran bit patterns."""
    from epsr26 import common
    from epsr26.common import ran1com
    from epsr26.library import auxiliary_routines
    out = {}
    for seed in (0, -1, -12345, -2147483647, 123, -987654321):
        common.reset()
        ran1com.idum = seed
        vals = [auxiliary_routines.ran1() for _ in range(3000)]
        key = f"seed_{seed}".replace("-", "m")
        out[key] = np.array(vals, dtype=np.float32)
        for k, v in refstate.ran1_state().items():
            out[key + "_after_" + k] = v
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
    # the reference's gfortran golden file (tests/library/data/ran1_reference.txt)
    path = os.path.join(REF, "tests/library/data/ran1_reference.txt")
    blocks = parse_ran1_reference(path)
    np.savez_compressed(os.path.join(HERE, "ran1_reference.npz"), **blocks)


def parse_ran1_reference(path):
    """Blocks of the gfortran ran1 golden file (tests/library/test_ran1.py:22-32): a header
    line ("seed N" or "continued"), 1000 int32 bit patterns of the real*4 deviates, then the
    saveran1 state line "mcall idum iy iv(1..32)"."""
    out = {}
    lines = open(path).read().splitlines()
    i = 0
    k = 0
    while i < len(lines):
        head = lines[i].strip()
        vals = [int(v) for v in lines[i + 1:i + 1001]]
        state = [int(v) for v in lines[i + 1001].split()]
        out[f"block{k}_header"] = np.array(head)
        out[f"block{k}_bits"] = np.array(vals, dtype=np.int64).astype(np.uint32)
        out[f"block{k}_state"] = np.array(state, dtype=np.int64)
        i += 1002
        k += 1
    out["nblocks"] = np.int32(k)
    return out


CASES = {
    "c1_water": lambda: run_case("c1_water", configs.c1_water(seed=1), cycles=2, ngrsamples=0),
    "c1_sampled": lambda: run_case("c1_sampled", configs.c1_water(seed=2), cycles=1, ngrsamples=30,
                                   transforms=False),
    "mix_small": lambda: run_case("mix_small", configs.c2_mixture(seed=3, ndmso=20, nwater=40), cycles=2,
                                  ngrsamples=0, nq=300, qstep=0.1),
    "silica": lambda: run_case("silica", configs.silica(seed=4, natom=240), cycles=2, ngrsamples=0,
                               transforms=False, wholerot=0.0),
    # a translation step far below the float32 spacing of the centres: movem's displacement
    # rounds away and its retry doubles the step until a centre moves (molfit.py:752-758)
    "c1_retry": lambda: run_case("c1_retry", configs.c1_water(seed=5), cycles=2, ngrsamples=0, transforms=False,
                                 wholetrans_A=1.0e-9),
    "c2_mixture": lambda: run_case("c2_mixture", configs.c2_mixture(seed=1), cycles=1, ngrsamples=0,
                                   transforms=False),
    "fitexp": lambda: run_fit(),
    "ran1": lambda: run_ran1(),
}


if __name__ == "__main__":
    refstate.load_reference(os.path.join(REF, "src"))
    names = sys.argv[1:] or list(CASES)
    for n in names:
        CASES[n]()
