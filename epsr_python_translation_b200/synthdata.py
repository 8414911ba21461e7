"""Synthetic neutron data sets produced by the method itself under a perturbed potential.

The workloads fit their empirical potential to data; no measured data set of these systems is
used, so the data are generated the way a known answer is made for a refinement test: the
plain Monte Carlo of this package (cell list, pair store, molfit sweeps, atogen, gensq on the
device) is run on the workload's box with its empirical potential scaled by 1.5, the
intermolecular partial S(Q) are averaged over samples, and each data set is their
combination with the set's neutron weights plus seeded Gaussian noise (sigma 0.005).

Weights.  For atom labels with neutron scattering lengths b (fm: H -3.739, D 6.671, C 6.646,
O 5.803, S 2.847) and atom fractions c, the weight of the pair (a, b) is
(2 - delta_ab) c_a c_b b_a b_b / (sum_i c_i b_i)^2.  C2 has three isotope contrasts: fully
deuterated, fully protiated and 50:50 H/D (every hydrogen's length the mean of H and D); C3
has one data set, heavy water.

    python -m epsr_python_translation_b200.synthdata [c2_mixture|c3_water ...]

writes data/<name>_data.npz (weights and data), which configs.make_workload reads; the
generation needs a B200.
"""

from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
DATA = os.path.join(HERE, "data")
B = {"H": -3.739, "D": 6.671, "C": 6.646, "O": 5.803, "S": 2.847}
CONTRASTS = {"c2_mixture": ("D", "H", "HD"), "c3_water": ("D",)}
SAMPLES = {"c2_mixture": (40, 10, 5), "c3_water": (20, 4, 5)}    # warm-up sweeps, samples, sweeps per sample


def element(label):
    return "S" if label.startswith("S") else label[:1].upper()


def neutron_weights(system, contrast):
    """(npairs,) float64 pair weights of one contrast ("D", "H" or "HD")."""
    def length(label):
        e = element(label)
        if e == "H":
            return {"D": B["D"], "H": B["H"], "HD": 0.5 * (B["H"] + B["D"])}[contrast]
        return B[e]
    b = np.array([length(lab) for lab in system.type_labels], np.float64)
    c = np.array(system.cfrac, np.float64)
    norm = float(np.sum(c * b)) ** 2
    w = np.zeros(system.npairs)
    for p in range(system.npairs):
        i, j = int(system.n1extr[p]), int(system.n2extr[p])
        w[p] = (1.0 if i == j else 2.0) * c[i] * c[j] * b[i] * b[j] / norm
    return w


def path(name):
    return os.path.join(DATA, f"{name}_data.npz")


def load(name):
    """(weights [ndata][npairs] float64, data [ndata][nq+1] float32) or None if not generated."""
    p = path(name)
    if not os.path.exists(p):
        return None
    z = np.load(p)
    return z["weights"], z["data"]


def generate(name, seed=1):
    import torch

    from . import configs, transforms
    from .box import BoxArrays, Ran1State, trsteps
    from .device import DeviceBox
    wl = configs.make_workload(name, seed=seed, data_source="analytic")
    s = wl.system
    box = BoxArrays.from_system(s)
    box.xavs = (box.xavs * np.float32(1.5)).astype(np.float32)     # the perturbed potential
    box.xavs1 = (box.xavs1 * np.float32(1.5)).astype(np.float32)
    d = DeviceBox(box)
    tmax, tmin = trsteps(box.natomr)
    d.mc_setup(rejrate=np.float32(0.75), stepr=1.0, stepm=1.0, wholerot=wl.wholerot, wholetrans=wl.wholetrans,
               ran1=Ran1State(idum=-(1000 + seed)), trstepmax=tmax, trstepmin=tmin)
    warm, nsamp, per = SAMPLES[name]
    d.cell_list(wl.nmolcell, box.sepmax)
    d.fmolec1(wl.eintra, strict=False)
    for k in range(warm):
        d.molfit(strict=False)
        if k % 10 == 9:                         # the store is rebuilt as the iteration loop does
            d.cell_list(wl.nmolcell, box.sepmax)
            d.fmolec1(wl.eintra, strict=False)
    ld = box.npt + 1
    foq = torch.from_numpy(np.ascontiguousarray(wl.foqols)).cuda()
    ycoh = torch.from_numpy(np.ascontiguousarray(wl.ycoh[:ld], np.float32)).cuda()
    nat = torch.ones(box.ntype, dtype=torch.float32, device="cuda")
    acc = None
    for _ in range(nsamp):
        d.cell_list(wl.nmolcell, box.sepmax)
        d.fmolec1(wl.eintra, strict=False)
        for _ in range(per):
            d.molfit(strict=False)
        d.atogen(wl.ngrsamples, d.m_ran1, np.full(box.npairs, -2.0, np.float32), ycoh=wl.ycoh)
        sofq = transforms.gensq(wl.nq, box.npt1, d.a_wav, ld, foq, wl.nq + 1, 1, ycoh, d.n2extr, nat, box.npairs)
        inter = sofq.view(2, box.npairs, wl.nq + 1)[1].double().cpu().numpy()
        acc = inter if acc is None else acc + inter
    d.check_status()
    inter = acc / nsamp
    rng = np.random.default_rng(seed + 500)
    ws = np.stack([neutron_weights(s, c) for c in CONTRASTS[name]])
    data = np.zeros((ws.shape[0], wl.nq + 1), np.float32)
    for k in range(ws.shape[0]):
        data[k, 1:] = (ws[k] @ inter[:, 1:] + rng.normal(0.0, 0.005, size=wl.nq)).astype(np.float32)
    os.makedirs(DATA, exist_ok=True)
    np.savez_compressed(path(name), weights=ws, data=data, contrasts=np.array(CONTRASTS[name]),
                        q=wl.q, ep_scale=np.float32(1.5), samples=np.array(SAMPLES[name]))
    return ws, data


if __name__ == "__main__":
    for n in sys.argv[1:] or ["c2_mixture", "c3_water"]:
        w, dd = generate(n)
        print(n, w.shape, dd.shape, float(np.abs(dd).max()))
