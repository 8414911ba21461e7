"""The EPSR iteration of the pair path on the CPU oracle (TEST INFRASTRUCTURE ONLY).

Used by bench.py's CPU-baseline leg and its reference arm: the same stages, inputs and
order as epsr_python_translation_b200.iteration.EpsrIteration, computed by the C
restatement of the reference (single-threaded, as the reference).
"""

from __future__ import annotations

import time

import numpy as np

from epsr_python_translation_b200.box import BoxArrays, Ran1State
from oracle import oracle

f32 = np.float32


class CpuIteration:
    def __init__(self, wl, ran1_seed=0):
        self.wl = wl
        self.box = BoxArrays.from_system(wl.system)
        b = self.box
        nmt = b.nmoltype
        self.mc = dict(rejrate=f32(wl.rejrate), stepr=f32(1.0), stepm=f32(1.0), wholerot=wl.wholerot.copy(),
                       wholetrans=wl.wholetrans.copy(), internrot=np.zeros(nmt, f32),
                       interntrans=np.zeros(nmt, f32), ireset=0, nstepreject=np.zeros(b.nmol, np.int32))
        self.ran1 = Ran1State(idum=ran1_seed)
        ndata = wl.data.shape[0]
        self.pwtold = [np.zeros(wl.nterms + 1, f32) for _ in range(ndata)]
        self.stepp = [f32(0.01)] * ndata
        self.rows = np.ascontiguousarray(wl.foqols.T)   # (nq+1, npt1+1)
        self.stage_s = {}
        self.pair_updates = 0
        self.nisum_mc, self.fadds, self.faddbs, self.ergold1 = 1, f32(0.0), f32(0.0), f32(0.0)
        self.rot = None
        if wl.rotfreq > 0:
            from epsr_python_translation_b200 import configs
            r = configs.rotations(wl.system)
            m = dict(configs.intra_model(wl.system), ngrot=r["ngrot"])
            self.rot = dict(model=m, nrf=r["nrf"], nrl=r["nrl"], axis=r["axis"].reshape(-1), first=r["first"],
                            last=r["last"], atoms=r["atoms"], stepri=f32(1.0), rotcycle=0, faddbs=f32(0.0))
            self.mc["ngrot"] = r["ngrot"]
            self.mc["internrot"] = np.array(wl.internrot, f32)
        ep = wl.ep
        if ep is not None:
            b = self.box
            self.pcoefp = np.array(ep.pcoefp, f32)
            self.ep_pwtold = np.zeros(wl.nterms + 1, f32)
            self.ep_tabs = {"xavs": b.xavs, "xavs1": b.xavs1, "xavtot": (b.ecoul + b.xavs).astype(f32),
                            "xavtot1": (b.ecoul1 + b.xavs1).astype(f32)}
            self.ep_par = np.array([ep.absolute_energy, ep.erequnit, ep.ereqstep, ep.potfacamp], f32)

    def step(self, stages=None, sample_sweeps=None):
        """One iteration.  sample_sweeps: run only that many of the iteration's molfit sweeps
        and charge the molfit stage their mean time x the iteration's sweep count (a bounded
        sample of a long iteration; stage_s then holds the extrapolated iteration)."""
        wl, b = self.wl, self.box
        nsw = wl.ntimes if not sample_sweeps else max(1, min(int(sample_sweeps), wl.ntimes))
        t = {}
        t0 = time.perf_counter()
        cells = oracle.cell_list(b, wl.nmolcell, b.sepmax)
        t["cells"] = time.perf_counter() - t0
        t0 = time.perf_counter()
        model = None
        if wl.intra > 0:
            from epsr_python_translation_b200 import configs
            model = configs.intra_model(wl.system)
        if self.rot is not None:
            model = self.rot["model"]
        st = oracle.fmolec1(b, cells, wl.eintra if model is None else oracle.en_mole_intra_all(b, model))
        t["fmolec1"] = time.perf_counter() - t0
        self.cells, self.st = cells, st
        t0 = time.perf_counter()
        for _ in range(nsw):
            if wl.intra > 0 and self.nisum_mc >= wl.intra:
                # molfit's intramolecular branch, then runepsr17's minimage and store rebuild
                self.fadds, self.faddbs, _, self.ergold1, self.ran1 = oracle.molfit_shake(
                    b, st, self.mc, model, wl.stepmi, self.ran1, self.fadds, self.faddbs, self.ergold1)
                self.nisum_mc = 1
                oracle.minimage_centres(b)
                st = oracle.fmolec1(b, cells, oracle.en_mole_intra_all(b, model))
            else:
                rot = self.rot
                if rot is not None:
                    rot["rotcycle"] = int(self.nisum_mc % wl.rotfreq == 0)
                    rot["faddbs"] = self.faddbs
                _, tr, self.ran1 = oracle.molfit(b, cells, st, self.mc, self.ran1, record_cos=False, rot=rot)
                if rot is not None:
                    self.faddbs = tr["faddbs"]
                self.nisum_mc += 1
        t["molfit"] = (time.perf_counter() - t0) * (wl.ntimes / nsw)
        self.sampled_sweeps = nsw
        if stages == "mc":
            self.stage_s = t
            return
        t0 = time.perf_counter()
        wav, potex, ngr, self.ran1 = oracle.atogen(b, wl.ngrsamples, self.ran1, np.full(b.npairs, -2.0, f32),
                                                   ycoh=wl.ycoh)
        t["atogen"] = time.perf_counter() - t0
        # pair-updates: a full (probaccept >= 1) histogram visits every atom pair once; a sampled
        # one visits, per origin molecule, its atoms against every other atom (counted here
        # with the mean molecule size), plus the intramolecular pairs of every molecule
        n_at = b.natom
        intra = int(sum(int(n) * (int(n) - 1) // 2 for n in b.nato))
        if ngr >= b.nmol:
            self.pair_updates = n_at * (n_at - 1) // 2
        else:
            self.pair_updates = intra + int(ngr * (n_at / b.nmol) * n_at)
        t0 = time.perf_counter()
        nq = wl.nq
        sofq = oracle.gensq(nq, b.npt1, wav, self.rows, wl.ycoh[: b.npt + 1], b.n2extr, np.ones(b.ntype, f32))
        t["gensq"] = time.perf_counter() - t0
        t0 = time.perf_counter()
        self.press = oracle.press(b, st, b.npt1, b.simt, f32(wl.system.L ** 3))
        t["press"] = time.perf_counter() - t0
        t0 = time.perf_counter()
        inter = sofq[1]
        dts = oracle.ptgnsq_difference(wl.data, wl.weights, inter)
        chis = []
        for k in range(wl.data.shape[0]):
            dt = dts[k]
            res, self.ran1 = oracle.fit_expansion(dt, wl.expr, self.pwtold[k], self.stepp[k], 1, nq, 1, wl.nterms,
                                                  1000, 10, self.ran1)
            self.pwtold[k] = res["wtold"]
            self.stepp[k] = res["stepr"]
            chis.append(float(res["chisq"]))
        self.chisq = chis
        self.wav, self.sofq = wav, sofq
        t["fit_expansion"] = time.perf_counter() - t0
        t0 = time.perf_counter()
        ep = wl.ep
        if ep is not None:
            # ptgnsq's coefficient increment, then generate_ep(.false.), which rebuilds its basis
            # on every call as the reference does; the next iteration's energies read the tables
            expgr = oracle.calc_pwrexpr_grad(b.npt2, wl.nterms, ep.pdmin, ep.pdstep, ep.pdmax, ep.psigma2, ep.rho, b.x,
                                             rbroad=ep.rbroad)
            self.pcoefp = oracle.ep_update(self.pcoefp, ep.iref, ep.efacp, wl.weights, np.stack(self.pwtold),
                                           ep.potfac)
            tabs, self.pcoefp, self.ep_pwtold, _, _, _ = oracle.generate_ep(
                b.npt, b.npt2, wl.nterms, expgr, self.pcoefp, ep.iref, b.dmax, b.xstar, ep.wfac, b.ecoul, self.ep_tabs,
                self.ep_pwtold, self.ep_par, ep.potfac, False)
            b.xavs[...] = tabs["xavs"]
            b.xavs1[...] = tabs["xavs1"]
            self.ep_tabs = {"xavs": b.xavs, "xavs1": b.xavs1, "xavtot": tabs["xavtot"], "xavtot1": tabs["xavtot1"]}
        t["ep"] = time.perf_counter() - t0
        t0 = time.perf_counter()
        self.nsum = getattr(self, "nsum", 0) + 1
        fc1 = float(f32(1.0) / f32(self.nsum))
        fc2 = float(f32(self.nsum - 1)) * fc1
        if not hasattr(self, "sums"):
            ld = b.npt + 1
            self.sums = {k: np.zeros((b.npairs, nq + 1), f32) for k in ("soqintra", "soqinter", "sq2intra", "sq2inter")}
            self.sums.update({k: np.zeros((b.npairs, ld), f32)
                              for k in ("gorintra", "gorinter", "gr2intra", "gr2inter", "entsig")})
        self.sums.update(oracle.sumsq(nq, sofq, fc1, fc2, self.sums))
        self.sums.update(oracle.sumgr(b.npt1, wav, wl.ycoh[: b.npt + 1], fc1, fc2, self.sums))
        t["sums"] = time.perf_counter() - t0
        t0 = time.perf_counter()
        r = b.x[: b.npt1 + 1].copy()
        oracle.stog(f32(b.natom / wl.system.L ** 3), wl.q, inter, r, np.full(b.npairs, 2, np.int32),
                    np.full(b.npairs, nq, np.int32), wl.xwt)
        t["stog"] = time.perf_counter() - t0
        self.stage_s = t

    def sweep(self):
        """One molfit sweep on the cell list and store of the last step (the reference does not
        rebuild them between the sweeps of an iteration)."""
        _, _, self.ran1 = oracle.molfit(self.box, self.cells, self.st, self.mc, self.ran1, record_cos=False)
