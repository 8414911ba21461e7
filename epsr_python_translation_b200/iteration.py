"""One EPSR iteration of the pair path on the device (the body of runepsr17's loop,
epsr_standalone_rev3.py:1235-1842, restricted to the hot path).

Per call of ``step()``: cell list (:1265), fmolec1 (:1280), ``ntimes`` molfit cycles
(:1314-1318), atogen (:1397), gensq (:1400), one fit_expansion per dataset on the
difference between data and the weighted simulated S(Q) (ptgnsq :3846-3944), and stog of
the simulated S(Q) (:1987).  All state stays on the GPU; per-stage device times are
recorded with CUDA events on the launching stream.
"""

from __future__ import annotations

import numpy as np
import torch

from . import transforms
from .box import BoxArrays, Ran1State, trsteps
from .configs import Workload
from .device import DeviceBox, press_scalars

f32 = np.float32
STAGES = ("cells", "fmolec1", "molfit", "atogen", "gensq", "press", "fit_expansion", "stog")


class EpsrIteration:
    def __init__(self, wl: Workload, device="cuda", strict=False, ran1_seed=0):
        self.wl = wl
        self.strict = strict
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
        self.weights = torch.from_numpy(np.ascontiguousarray(wl.weights, dtype=np.float32)).to(dev)
        self._dt = torch.empty_like(self.data)
        self.natomsphere = torch.ones(b.ntype, dtype=torch.float32, device=dev)
        self.rminex = torch.full((b.npairs,), -2.0, dtype=torch.float32, device=dev)
        self.xwt = torch.from_numpy(wl.xwt).to(dev)
        ndata = wl.data.shape[0]
        self.pwtold = torch.zeros(ndata, wl.nterms + 1, dtype=torch.float32, device=dev)
        self.stepp = np.full(ndata, f32(0.01), f32)
        self._fit_scratch = torch.empty(4096, dtype=torch.uint8, device=dev)
        self.r = torch.from_numpy(b.x[: b.npt1 + 1].copy()).to(dev)
        self.nqmin = torch.full((b.npairs,), 2, dtype=torch.int32, device=dev)
        self.nqmax = torch.full((b.npairs,), wl.nq, dtype=torch.int32, device=dev)
        self.events = {k: (torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
                       for k in STAGES}
        self.moves_per_step = wl.ntimes * b.nmol
        self.volume = f32(float(wl.system.L) ** 3)          # box volume (A^3) for press
        self.pair_updates = 0
        self.fit_trials = 0

    def _mark(self, stage, end=False):
        self.events[stage][1 if end else 0].record()

    def step(self):
        wl, d, b = self.wl, self.d, self.box
        self._mark("cells")
        d.cell_list(wl.nmolcell, b.sepmax)
        self._mark("cells", True)
        self._mark("fmolec1")
        self.ftest = d.fmolec1(wl.eintra, strict=self.strict)
        self._mark("fmolec1", True)
        self._mark("molfit")
        for _ in range(wl.ntimes):
            d.molfit(strict=self.strict)
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
        self.fit_trials = int(res["trials"].sum())
        self._mark("fit_expansion", True)
        self._mark("stog")
        self.gofr = transforms.stog(float(b.natom) / float(wl.system.L) ** 3, self.q, inter, self.r, self.nqmin,
                                    self.nqmax, self.xwt)
        self._mark("stog", True)

    def stage_ms(self):
        torch.cuda.synchronize()
        return {k: self.events[k][0].elapsed_time(self.events[k][1]) for k in STAGES}

    # ------------------------------------------------------------------ host boundary
    def upload_inputs(self, coords):
        """Host -> device copy of the coordinates (the per-iteration input of the loop)."""
        self.d.upload_coords(*coords)

    def download_outputs(self):
        """Device -> host copy of what the host consumers of the loop read after an
        iteration: coordinates (.ato writer), the histograms (sumgr) and the EP
        coefficients (generate_ep).  Returns the arrays and their total bytes."""
        co = self.d.download_coords()
        wav = self.d.a_wav.cpu().numpy()
        pw = self.pwtold.cpu().numpy()
        nbytes = sum(v.nbytes for v in co.values()) + wav.nbytes + pw.nbytes
        return (co, wav, pw), nbytes
