"""One EPSR iteration of the pair path on the device (the body of runepsr17's loop,
epsr_standalone_rev3.py:1235-1842, restricted to the hot path).

Per call of ``step()``: cell list (:1265), fmolec1 (:1280), ``ntimes`` molfit cycles
(:1314-1318), atogen (:1397), gensq (:1400), press (:1655), one fit_expansion per dataset on
the difference between data and the weighted simulated S(Q) (ptgnsq :3846-3944), the EP
refinement that follows the fits when the workload has one (ptgnsq :3948-3962, generate_ep
:4014; the next iteration's energies use the refined tables), the running averages
(:1611-1642) and stog of the simulated S(Q) (:1987).  All state stays on the GPU; per-stage device times are
recorded with CUDA events on the launching stream.
"""

from __future__ import annotations

import numpy as np
import torch

import ctypes as C

from . import _lib, potential, transforms
from .box import BoxArrays, Ran1State, trsteps
from .configs import Workload
from .device import DeviceBox, press_scalars

f32 = np.float32
STAGES = ("cells", "fmolec1", "molfit", "atogen", "gensq", "press", "fit_expansion", "ep", "sums", "stog")


class EpsrIteration:
    def __init__(self, wl: Workload, device="cuda", strict=False, ran1_seed=0, native=False):
        self.wl = wl
        self.strict = strict
        self.native = native          # steps after the first through epsr_iteration_step
        self._plan = None
        self.box = BoxArrays.from_system(wl.system)
        self.d = DeviceBox(self.box, device=device)
        b = self.box
        tmax, tmin = trsteps(b.natomr)
        self.d.mc_setup(rejrate=wl.rejrate, stepr=1.0, stepm=1.0, wholerot=wl.wholerot, wholetrans=wl.wholetrans,
                        ran1=Ran1State(idum=ran1_seed), trstepmax=tmax, trstepmin=tmin)
        self.ran1 = self.d.m_ran1        # one stream shared by molfit, atogen and fit_expansion
        dev = self.d.dev
        self.q = torch.from_numpy(wl.q).to(dev)
        self.foqols = torch.from_numpy(np.ascontiguousarray(wl.foqols)).to(dev)
        self.ycoh = torch.from_numpy(np.ascontiguousarray(wl.ycoh[: b.npt + 1], f32)).to(dev)
        self.expr = torch.from_numpy(wl.expr).to(dev)
        self.data = torch.from_numpy(wl.data).to(dev)
        # the data-set weights cwt (and the potential weights cwtpot, the same here) are real*8
        self.weights = torch.from_numpy(np.ascontiguousarray(wl.weights, dtype=np.float64)).to(dev)
        self._dt = torch.empty_like(self.data)
        self.natomsphere = torch.ones(b.ntype, dtype=torch.float32, device=dev)
        self.rminex = torch.full((b.npairs,), -2.0, dtype=torch.float32, device=dev)
        self.xwt = torch.from_numpy(wl.xwt).to(dev)
        ndata = wl.data.shape[0]
        self.pwtold = torch.zeros(ndata, wl.nterms + 1, dtype=torch.float32, device=dev)
        self.stepp = np.full(ndata, f32(0.01), f32)
        self._fit_scratch = torch.empty(4096, dtype=torch.uint8, device=dev)
        # running averages of S(Q) and g(r) with their error bars (epsr16 soq*/sq2*, gor*/gr2*,
        # entsig), accumulated every iteration as runepsr17 does (:1611-1642)
        self.nsum = 0
        self.sums_sq = {k: torch.zeros(b.npairs, wl.nq + 1, dtype=torch.float32, device=dev)
                        for k in transforms.SQ_ARRAYS}
        self.sums_gr = {k: torch.zeros(b.npairs, b.npt + 1, dtype=torch.float32, device=dev)
                        for k in transforms.GR_ARRAYS}
        self.r = torch.from_numpy(b.x[: b.npt1 + 1].copy()).to(dev)
        self.nqmin = torch.full((b.npairs,), 2, dtype=torch.int32, device=dev)
        self.nqmax = torch.full((b.npairs,), wl.nq, dtype=torch.int32, device=dev)
        self.ep = wl.ep
        if self.ep is not None:
            self._ep_setup()
        # flexible molecules: intramolecular cycles every wl.intra molfit cycles (molfit.py:124)
        self.intra_model = None
        self.nisum_mc = 1
        self.rot = None
        if wl.intra > 0 or wl.rotfreq > 0:
            from . import configs
            from .intra import IntraModel
            self.rot = configs.rotations(wl.system) if wl.rotfreq > 0 else None
            ngrot = self.rot["ngrot"] if self.rot is not None else None
            self.intra_model = IntraModel(self.d, **configs.intra_model(wl.system), ngrot=ngrot)
            self.faddbs = torch.zeros(1, dtype=torch.float32, device=dev)
            self._eintra_work = torch.zeros(b.nmol, dtype=torch.float32, device=dev)
            self._nmovei = torch.zeros(2 * b.nmoltype, dtype=torch.int32, device=dev)
        if self.rot is not None:
            # internal rotations of the templates' ROT groups every rotfreq whole-molecule cycles
            # (molfit.py:295-360), the intramolecular change accumulated in faddbs
            r = self.rot
            self.d.set_rotations(self.intra_model, r["nrf"], r["nrl"], r["axis"], r["first"], r["last"], r["atoms"],
                                 stepri=1.0, faddbs=0.0)
            self.d.m_internrot.copy_(torch.from_numpy(wl.internrot))
        self.events = {k: (torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
                       for k in STAGES}
        self.moves_per_step = wl.ntimes * b.nmol
        self.volume = f32(float(wl.system.L) ** 3)          # box volume (A^3) for press
        self.pair_updates = 0
        self.fit_trials = 0

    def _ep_setup(self):
        """Device state of the EP refinement: the r-space basis (built once on the host; the
        reference rebuilds the same matrix inside every generate_ep call), the coefficient
        sets, the unpacked tables and the potential factor.  A refined EP's gradient is
        nonzero at the last table point, so the energies read the tables up to npt2."""
        ep, b, d, wl = self.ep, self.box, self.d, self.wl
        dev = d.dev
        t = lambda a: torch.from_numpy(np.ascontiguousarray(a, f32)).to(dev)  # noqa: E731
        expgr, _ = potential.basis(b.npt2, wl.nterms, b.x, False, ep.pdmin, ep.pdstep, ep.pdmax, ep.psigma2, ep.rho,
                                   ep.rbroad)
        self.ep_expgr = t(expgr)
        self.ep_pcoefp = t(ep.pcoefp)
        self.ep_iref = np.ascontiguousarray(ep.iref, np.int32)
        self.ep_efacp = t(ep.efacp)
        self.ep_wfac = t(ep.wfac)
        self.ep_ecoul, self.ep_ecoul1 = t(b.ecoul), t(b.ecoul1)
        self.ep_tabs = {"xavs": t(b.xavs), "xavs1": t(b.xavs1), "xavtot": t(b.ecoul + b.xavs),
                        "xavtot1": t(b.ecoul1 + b.xavs1)}
        self.ep_pwtold = torch.zeros(wl.nterms + 1, dtype=torch.float32, device=dev)
        self.ep_potfac = t([ep.potfac])
        self.ep_result = torch.zeros(2, dtype=torch.float32, device=dev)
        d.izcut = b.npt2
        d.cbox.izcut = b.npt2

    def _ep_refine(self):
        ep, b, d, wl = self.ep, self.box, self.d, self.wl
        potential.ep_update(self.ep_pcoefp, self.ep_iref, self.ep_efacp, self.weights, self.pwtold, ep.potfac)
        potential.generate_ep(b.npt, b.npt2, wl.nterms, self.ep_expgr, self.ep_pcoefp, self.ep_iref, b.dmax, d.xstar,
                              self.ep_wfac, self.ep_ecoul, self.ep_tabs, self.ep_pwtold, ep.absolute_energy,
                              ep.erequnit, ep.ereqstep, ep.potfacamp, self.ep_potfac, changepotfac=False,
                              result=self.ep_result)
        potential.pack_tables(self.ep_tabs["xavs"], self.ep_tabs["xavs1"], self.ep_ecoul, self.ep_ecoul1, d.tab)

    def _mark(self, stage, end=False):
        self.events[stage][1 if end else 0].record()

    def step(self):
        if self.native and self._plan is not None:
            try:
                return self._step_native()
            except _lib.EpsrGpuError as e:
                if e.code != 3:             # capacity: this iteration sizes its buffers below
                    raise
                self._plan = None
        self._step_python()
        if self.native:
            self._build_plan()

    def _step_python(self):
        wl, d, b = self.wl, self.d, self.box
        self._mark("cells")
        d.cell_list(wl.nmolcell, b.sepmax)
        self._mark("cells", True)
        self._mark("fmolec1")
        eintra = wl.eintra if self.intra_model is None else self.intra_model.en_mole_intra(self._eintra_work)
        self.ftest = d.fmolec1(eintra, strict=self.strict)
        self._mark("fmolec1", True)
        self._mark("molfit")
        for _ in range(wl.ntimes):
            if wl.intra > 0 and self.nisum_mc >= wl.intra:
                # molfit's intramolecular branch, then runepsr17's minimage and store rebuild
                self._nmovei.copy_(self.intra_model.molfit_shake(wl.stepmi, self.faddbs))
                self.nisum_mc = 1
                d.minimage_centres()
                self.ftest = d.fmolec1(self.intra_model.en_mole_intra(self._eintra_work), strict=self.strict)
            else:
                d.molfit(strict=self.strict, rotcycle=wl.rotfreq > 0 and self.nisum_mc % wl.rotfreq == 0)
                self.nisum_mc += 1
        self._mark("molfit", True)
        self._mark("atogen")
        d.atogen(wl.ngrsamples, self.ran1, self.rminex, ycoh=self.ycoh)
        self.pair_updates = d.last_pair_updates
        self._mark("atogen", True)
        self._mark("gensq")
        nq = wl.nq
        ld = b.npt + 1
        sofq = transforms.gensq(nq, b.npt1, d.a_wav, ld, self.foqols, nq + 1, 1, self.ycoh, d.n2extr,
                                self.natomsphere, b.npairs)
        self.sofq = sofq.view(2, b.npairs, nq + 1)
        inter = self.sofq[1]                                   # (npairs, nq+1)
        # per data set: the difference between the data and the weighted simulated S(Q)
        dt = transforms.ptgnsq_difference(self.data, self.weights, inter, out=self._dt)   # (ndata, nq+1)
        self._mark("gensq", True)
        self._mark("press")
        sumc, presst = d.press(b.npt1, strict=self.strict)
        self.energy, self.pressc = press_scalars(b.nmol, sumc, presst, b.simt, self.volume)
        self._mark("press", True)
        self._mark("fit_expansion")
        res = transforms.fit_expansion_batch(dt, self.expr, self.pwtold, self.stepp, 1, nq, 1, wl.nterms, 1000, 10,
                                             self.ran1, strict=self.strict, scratch=self._fit_scratch)
        self.pwtold = res["wtold"]
        self.stepp = res["stepr"]
        self.chisq = res["chisq"]
        self.fit_trials = int(res["trials"].sum())
        self._mark("fit_expansion", True)
        self._mark("ep")
        if self.ep is not None:
            self._ep_refine()
        self._mark("ep", True)
        self._mark("sums")
        self.nsum += 1
        fc1 = float(np.float32(1.0) / np.float32(self.nsum))
        fc2 = float(np.float32(self.nsum - 1)) * fc1
        transforms.sumsq(nq, sofq, fc1, fc2, self.sums_sq)
        transforms.sumgr(b.npt1, d.a_wav, self.ycoh, fc1, fc2, self.sums_gr)
        self._mark("sums", True)
        self._mark("stog")
        self.gofr = transforms.stog(float(b.natom) / float(wl.system.L) ** 3, self.q, inter, self.r, self.nqmin,
                                    self.nqmax, self.xwt)
        self._mark("stog", True)

    # ------------------------------------------------------------------ native driver
    def _build_plan(self):
        """The epsr_iteration_t of this box, on the buffers the Python step sized (device
        tensors kept on self so the pointers stay valid)."""
        wl, d, b = self.wl, self.d, self.box
        nq, ld = wl.nq, b.npt + 1
        ndata = self.data.shape[0]
        dev = d.dev
        P = lambda t: C.c_void_p(t.data_ptr())
        it = _lib.Iteration()
        it.box = C.cast(C.pointer(d.cbox), C.c_void_p)
        it.mc = C.cast(C.pointer(d.cmc), C.c_void_p)
        it.nmolcell, it.rmax = wl.nmolcell, float(np.float32(b.sepmax))
        for i in range(6):
            it.lat6[i] = float(b.lat6[i])
        for i in range(9):
            it.lat9[i] = float(np.asarray(b.lat9, np.float32).reshape(-1)[i])
        it.cell_molcellno, it.cell_start, it.cell_mols, it.cell_offsets = (
            P(t) for t in (d.c_molcellno, d.c_start, d.c_mols, d.c_off))
        it.cell_scratch, it.cell_scratch_n = P(d._c_scr), d._c_scr.numel()
        it.store_m = d.s_mol.numel() // b.nmol
        it.store_capacity = d.s_erg.numel()
        it.nergpairm, it.molergpair, it.ergpairref, it.mirror, it.nergpair, it.ergpair = (
            P(t) for t in (d.s_nergpairm, d.s_mol, d.s_ref, d.s_mirror, d.s_n, d.s_erg))
        it.eintra = P(d.eintra)
        it.ntimes = wl.ntimes
        it.npt1, it.natomr, it.ngrsamples = b.npt1, b.natomr, wl.ngrsamples
        it.sizefactor, it.dmax = 1.0, float(b.dmax)
        self._n_wav = torch.zeros(2 * b.npairs * ld, dtype=torch.float32, device=dev)
        self._n_potex = torch.zeros(b.npairs, dtype=torch.float32, device=dev)
        self._n_counts = torch.zeros(2 * b.npairs * ld + b.npairs, dtype=torch.int64, device=dev)
        it.rminex, it.cfrac, it.ycoh, it.n1extr, it.n2extr = (
            P(t) for t in (self.rminex, d.cfrac, self.ycoh, d.n1extr, d.n2extr))
        it.wav, it.ldw, it.potex, it.counts = P(self._n_wav), ld, P(self._n_potex), P(self._n_counts)
        self._n_sofq = torch.zeros(2 * b.npairs * (nq + 1), dtype=torch.float32, device=dev)
        it.nq, it.ndata = nq, ndata
        it.foqols, it.foqols_sj, it.foqols_si = P(self.foqols), nq + 1, 1
        it.natomsphere, it.sofq = P(self.natomsphere), P(self._n_sofq)
        it.data, it.cwt, it.dt = P(self.data), P(self.weights), P(self._dt)
        self._n_wt = torch.zeros(ndata, wl.nterms + 1, dtype=torch.float32, device=dev)
        self._n_wtold = self.pwtold.clone()
        self._n_yout = torch.zeros(ndata, nq + 1, dtype=torch.float32, device=dev)
        self._n_scal = np.zeros((ndata, 4), np.float32)
        self._n_trials = np.zeros(ndata, np.int64)
        it.expr, it.nterms, it.ncfirst, it.nits, it.nfreq = P(self.expr), wl.nterms, 1, 1000, 10
        it.fit_wt, it.fit_wtold, it.fit_yout = P(self._n_wt), P(self._n_wtold), P(self._n_yout)
        it.fit_scal_host = self._n_scal.ctypes.data_as(C.c_void_p)
        it.fit_trials_host = self._n_trials.ctypes.data_as(C.c_void_p)
        self._n_gofr = torch.zeros(b.npairs, self.r.numel(), dtype=torch.float32, device=dev)
        it.rho = float(np.float32(float(b.natom) / float(wl.system.L) ** 3))
        it.q, it.r, it.nr = P(self.q), P(self.r), self.r.numel() - 1
        it.nqmin, it.nqmax, it.xwt, it.gofr = P(self.nqmin), P(self.nqmax), P(self.xwt), P(self._n_gofr)
        it.soqintra, it.soqinter, it.sq2intra, it.sq2inter = (P(self.sums_sq[k]) for k in transforms.SQ_ARRAYS)
        it.gorintra, it.gorinter, it.gr2intra, it.gr2inter, it.entsig = (
            P(self.sums_gr[k]) for k in transforms.GR_ARRAYS)
        if self.ep is not None:
            ep = self.ep
            it.refine = 1
            it.pcoefp, it.nsets, it.ldc = P(self.ep_pcoefp), self.ep_pcoefp.shape[0], self.ep_pcoefp.shape[1]
            it.irefpcof_host = self.ep_iref.ctypes.data_as(C.c_void_p)
            it.efacp, it.cwtpot, it.expgr, it.wfac = P(self.ep_efacp), P(self.weights), P(self.ep_expgr), P(self.ep_wfac)
            it.ecoul, it.ecoul1 = P(self.ep_ecoul), P(self.ep_ecoul1)
            it.xavs, it.xavs1, it.xavtot, it.xavtot1 = (P(self.ep_tabs[k]) for k in potential.TABLES)
            it.ep_pwtold, it.potfac, it.ep_result = P(self.ep_pwtold), P(self.ep_potfac), P(self.ep_result)
            it.pfact, it.absolute_energy, it.erequnit = ep.potfac, ep.absolute_energy, ep.erequnit
            it.ereqstep, it.potfacamp = ep.ereqstep, ep.potfacamp
            it.tab = P(d.tab)
        if self.intra_model is not None:
            it.intra, it.stepmi = wl.intra, float(f32(wl.stepmi))
            it.intra_model = C.cast(C.pointer(self.intra_model.c), C.c_void_p)
            it.faddbs, it.eintra_work, it.nmovei = P(self.faddbs), P(self._eintra_work), P(self._nmovei)
        it.strict = 1 if self.strict else 0
        it.rotfreq = wl.rotfreq if self.rot is not None else 0
        for k, name in enumerate(STAGES):       # the Python step has created these events
            it.stage_events[2 * k] = self.events[name][0].cuda_event
            it.stage_events[2 * k + 1] = self.events[name][1].cuda_event
        nb = int(d.lib.epsr_iteration_scratch_bytes(C.byref(it)))
        self._n_scratch = torch.empty(max(nb, 256), dtype=torch.uint8, device=dev)
        it.scratch, it.scratch_bytes = P(self._n_scratch), self._n_scratch.numel()
        self._plan = it
        self._rep = _lib.IterationReport()

    def _step_native(self):
        wl, b = self.wl, self.box
        self._n_scal[:, 0] = self.stepp
        self._plan.nsum = self.nsum + 1
        self._plan.nisum = self.nisum_mc
        _lib.check(self.d.lib.epsr_iteration_step(C.byref(self._plan), C.byref(self._rep),
                                                  C.c_void_p(torch.cuda.current_stream().cuda_stream)))
        r = self._rep
        self.d.nnbrefmax = int(r.nnbrefmax)
        if self.intra_model is not None or self.rot is not None:
            self.nisum_mc = int(r.nisum)
        if self.d.store is not None:        # the store struct other calls take follows the driver's layout
            self.d.store.nnbrefmax = int(r.nnbrefmax)
        self.ftest = (np.float32(r.ftest[0]), np.float32(r.ftest[1]))
        self.pair_updates = int(r.pair_updates)
        self.energy, self.pressc = press_scalars(b.nmol, np.float32(r.press[0]), float(r.press[1]), b.simt,
                                                 self.volume)
        self.pwtold = self._n_wtold
        self.stepp = self._n_scal[:, 0].copy()
        self.fit_trials = int(self._n_trials.sum())
        self.nsum += 1
        self.sofq = self._n_sofq.view(2, b.npairs, wl.nq + 1)
        self.gofr = self._n_gofr

    def stage_ms(self):
        torch.cuda.synchronize()
        return {k: self.events[k][0].elapsed_time(self.events[k][1]) for k in STAGES}

    # ------------------------------------------------------------------ host boundary
    def upload_inputs(self, coords):
        """Host -> device copy of the coordinates (the per-iteration input of the loop)."""
        self.d.upload_coords(*coords)

    def download_outputs(self):
        """Device -> host copy of what the host consumers of the loop read after an
        iteration: coordinates (.ato writer), the histograms of this iteration and the EP
        coefficients (the refined pcoefp when the EP is refined, else the fits' coefficients).
        Returns the arrays and their total bytes."""
        co = self.d.download_coords(stream_only=True)   # this box's stream only
        native = self.native and self._plan is not None
        wav = (self._n_wav if native else self.d.a_wav).cpu().numpy()
        pw = (self.ep_pcoefp if self.ep is not None else self.pwtold).cpu().numpy()
        nbytes = sum(v.nbytes for v in co.values()) + wav.nbytes + pw.nbytes
        return (co, wav, pw), nbytes
