"""Delayed-acceptance Monte Carlo with a learned first stage, over many boxes at once.

The plain method accepts a whole-molecule move with probability min(1, exp(-beta dE))
(molfit.py:401-408), where dE needs every pair energy of the moved molecule.  Here a small
network first screens the move from cheap features -- the radial histograms of the moved
molecule's neighbours within 8 A, 64 bins x 10 element-pair classes, before and after the
move -- with probability min(1, exp(-s)), s the network's antisymmetric estimate of beta dE
(s(before, after) = -s(after, before) by construction: s = (g(f, f') - g(f', f))/2); only a
move that passes is evaluated exactly and accepted with min(1, exp(-(beta dE - s))).  The two
stages together satisfy detailed balance with the plain test's distribution whatever s is, so
the surrogate changes only how much exact work a move costs, never what is sampled.

The network (surrogate.SurrogateNet: 1280 -> 128 -> 128 -> 1, SiLU, BF16 weights, FP32
accumulation, hand-written tcgen05 kernels) is trained on (features, beta dE) pairs that the
plain batched run records, with a held-out split; when the held-out RMS error (estimates and
targets clipped at ``TARGET_CLIP``, beyond which both stages reject anyway) exceeds
``RMSE_BOUND`` (in units of kT) the plain single-stage path takes over.

The boxes advance by the batched checkerboard scheme of batch.BatchBoxes, each sweep replayed
from a CUDA graph.  The effective sample size of each box's total-energy series is estimated
from its integrated autocorrelation time (Sokal's automatic window).
"""

from __future__ import annotations

import time

import numpy as np
import torch

from .batch import FEAT_IN, BatchBoxes
from .surrogate import SurrogateNet

RMSE_BOUND = 2.0        # kT: above this held-out error the plain single-stage path runs
TARGET_CLIP = 12.0      # kT: targets (and, for the held-out error, estimates) are clipped here:
                        # beyond it both stages reject with probability above 1 - 6e-6


def integrated_time(x, c=5.0):
    """Integrated autocorrelation time tau = 1 + 2 sum_t rho(t) of a series, with Sokal's
    automatic window (the smallest M with M >= c tau(M)); ESS = len(x) / tau."""
    x = np.asarray(x, np.float64)
    n = x.size
    if n < 4 or np.var(x) == 0:
        return 1.0
    y = x - x.mean()
    f = np.fft.rfft(y, 2 * n)
    acf = np.fft.irfft(f * np.conj(f))[:n]
    rho = acf / acf[0]
    taus = 2.0 * np.cumsum(rho) - 1.0
    for m in range(1, n):
        if m >= c * taus[m]:
            return float(max(taus[m], 1.0))
    return float(max(taus[-1], 1.0))


def ess(series):
    """Effective sample size of every column (box) of series [samples][boxes]; and the taus."""
    taus = np.array([integrated_time(series[:, b]) for b in range(series.shape[1])])
    return series.shape[0] / taus, taus


class LearnedMC:
    """B boxes advanced together; plain, recording and delayed-acceptance sweeps."""

    def __init__(self, systems, rot_deg=10.0, trans_A=0.5, seed=1, device="cuda", net_seed=0):
        self.bb = BatchBoxes(systems, rot_deg=rot_deg, trans_A=trans_A, seed=seed, device=device)
        self.dev = self.bb.dev
        self.net = SurrogateNet(device=device, seed=net_seed)
        self.fallback = False
        self.heldout_rmse = None
        self.bb.total_energy()

    # ------------------------------------------------------------------ data
    def collect(self, npairs, max_sweeps=50):
        """Record plain sweeps until at least npairs valid (features, beta dE) pairs exist.
        Returns x [2 n][1280] BF16 (rows 2q, 2q+1 = pair q's two orders) and t [n] FP32."""
        bb = self.bb
        per = bb.steps_per_sweep * bb.nslot
        nsw = max(1, min(max_sweeps, int(np.ceil(npairs / max(per * 0.5, 1)))))
        xs, ts = [], []
        have = 0
        for _ in range(max_sweeps):
            rec = {"x": torch.empty(2 * per, FEAT_IN, dtype=torch.bfloat16, device=self.dev),
                   "t": torch.empty(per, dtype=torch.float32, device=self.dev), "n": 0}
            bb.sweep("record", record=rec)
            ok = torch.isfinite(rec["t"])
            idx = torch.nonzero(ok).squeeze(1)
            rows = torch.stack([2 * idx, 2 * idx + 1], 1).reshape(-1)
            xs.append(rec["x"][rows])
            ts.append(rec["t"][idx])
            have += int(idx.numel())
            del rec
            if have >= npairs:
                break
        del nsw
        x = torch.cat(xs)
        t = torch.cat(ts)
        return x, t

    # ------------------------------------------------------------------ training
    def train(self, x, t, epochs=4, batch=2048, lr=1e-3, heldout=0.05, seed=0):
        """Adam on the pairs (clipped targets), a held-out fraction kept aside, the learning
        rate decayed over the epochs on a half cosine; returns dict with the loss per epoch and
        the held-out RMS error of s (kT).  Batches are contiguous runs of pairs after one random
        permutation."""
        npairs = t.numel()
        g = torch.Generator(device="cpu").manual_seed(seed)
        perm = torch.randperm(npairs, generator=g).to(self.dev)
        nho = max(int(heldout * npairs), batch // 2)
        ntr = ((npairs - nho) // (batch // 2)) * (batch // 2)
        tr, ho = perm[:ntr], perm[ntr:ntr + nho]
        rows_tr = torch.stack([2 * tr, 2 * tr + 1], 1).reshape(-1)
        xtr = x[rows_tr].contiguous()
        ttr = t[tr].clamp(-TARGET_CLIP, TARGET_CLIP).contiguous()
        xtt = xtr.t().contiguous()
        loss = torch.zeros(1, dtype=torch.float32, device=self.dev)
        nb = ntr // (batch // 2)
        hist = []
        t0 = time.perf_counter()
        for ep in range(epochs):
            tot = 0.0
            order = torch.randperm(nb, generator=g).tolist()
            acc = torch.zeros(1, dtype=torch.float64, device=self.dev)
            lr_ep = lr * 0.5 * (1.0 + np.cos(np.pi * ep / max(epochs, 1)))
            for bi in order:
                self.net.train_step(xtr, xtt, bi * batch, batch, ttr, lr_ep, loss=loss)
                acc += loss.double()
            tot = float(acc.item()) / ntr
            hist.append(tot)
        torch.cuda.synchronize()
        train_s = time.perf_counter() - t0
        self.net.check_status()
        rmse = self.heldout_error(x, t, ho)
        self.heldout_rmse = rmse
        self.fallback = not (rmse <= RMSE_BOUND)
        return {"loss_per_epoch": hist, "heldout_rmse_kT": rmse, "pairs_train": int(ntr), "pairs_heldout": int(nho),
                "train_s": train_s, "fallback": self.fallback}

    def surrogate(self, x):
        """s for every pair of rows (2q, 2q+1) of x."""
        rows = x.shape[0]
        y = self.net.forward(x)
        return 0.5 * (y[0:rows:2] - y[1:rows:2])

    def heldout_error(self, x, t, idx):
        rows = torch.stack([2 * idx, 2 * idx + 1], 1).reshape(-1)
        xh = x[rows].contiguous()
        s = self.surrogate(xh).clamp(-TARGET_CLIP, TARGET_CLIP)
        tt = t[idx].clamp(-TARGET_CLIP, TARGET_CLIP)
        return float(torch.sqrt(torch.mean((s - tt) ** 2)).item())

    # ------------------------------------------------------------------ sampling
    def run(self, sweeps, mode="plain"):
        """Replay `sweeps` sweeps of one mode from a CUDA graph; returns the energy series
        [sweeps+1][boxes] (kJ/mol), the device time (ms) and the counter deltas [boxes][4]
        (attempts, first-stage accepts, accepts, left-cell)."""
        if mode == "da" and self.fallback:
            mode = "plain"
        bb = self.bb
        g = bb.graphs.get(mode) or bb.capture(mode, self.net if mode == "da" else None)
        series = torch.zeros(sweeps + 1, bb.nbox, dtype=torch.float64, device=self.dev)
        series[0] = bb.energy
        c0 = bb.counters.clone()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for i in range(sweeps):
            g.replay()
            series[i + 1] = bb.energy
        e1.record()
        torch.cuda.synchronize()
        bb.check_status()
        self.net.check_status()
        cnt = (bb.counters - c0).cpu().numpy().reshape(bb.nbox, 4)
        return series.cpu().numpy(), e0.elapsed_time(e1), cnt, mode

    def residual_rmse(self):
        """RMS of beta dE - s over the moves of the last DA step that passed the first stage."""
        r = self.bb.resid
        if r is None:     # no delayed-acceptance step has run
            return None
        r = r[torch.isfinite(r)]
        return float(torch.sqrt(torch.mean(r * r)).item()) if r.numel() else None
