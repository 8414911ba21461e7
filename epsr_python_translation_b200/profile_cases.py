"""Small, self-contained runs of single kernels for profiling with Nsight Compute.

    python -m epsr_python_translation_b200.profile_cases <case> [repeats]

Each case builds its workload, runs a few untimed warm-up launches and then `repeats` (default
1) launches of the kernel of interest, so a capture such as

    ncu --set full --clock-control none -k regex:spec_energy -s 3 -c 1 \\
        python -m epsr_python_translation_b200.profile_cases c3_molfit

sees a representative launch after warm-up.  Cases:
  c3_molfit   one speculative molfit sweep of configuration C3 (20,000 water): spec_energy,
              spec_corr, spec_resolve
  c3_atogen   atogen of C3 over 1,000 sampled origins: ag_inter
  c5_batch    steps of 16 C5 boxes (2,700 DMSO + 5,300 water each) with the learned first
              stage: bmc_propose (features), umma_gemm (network), bmc_decide
  c4_hist     the all-pairs histograms of the 64 C4 boxes: bmc_hist_inter
"""

from __future__ import annotations

import sys

import numpy as np
import torch


def c3_molfit(rep):
    from . import configs
    from .box import BoxArrays, Ran1State, trsteps
    from .device import DeviceBox
    wl = configs.make_workload("c3_water", ntimes=1)
    box = BoxArrays.from_system(wl.system)
    d = DeviceBox(box)
    d.cell_list(wl.nmolcell, box.sepmax)
    d.fmolec1(wl.eintra, strict=False)
    tmax, tmin = trsteps(box.natomr)
    d.mc_setup(rejrate=np.float32(0.75), stepr=1.0, stepm=1.0, wholerot=wl.wholerot, wholetrans=wl.wholetrans,
               ran1=Ran1State(idum=-3), trstepmax=tmax, trstepmin=tmin)
    for _ in range(3 + rep):
        d.molfit(strict=False)
    torch.cuda.synchronize()
    d.check_status()


def c3_atogen(rep):
    from . import configs
    from .box import BoxArrays, Ran1State
    from .device import DeviceBox
    wl = configs.make_workload("c3_water", ntimes=1)
    box = BoxArrays.from_system(wl.system)
    d = DeviceBox(box)
    t = d.ran1_tensor(Ran1State(idum=-4))
    for _ in range(3 + rep):
        d.atogen(1000, t, np.full(box.npairs, -2.0, np.float32))
    torch.cuda.synchronize()


def c5_batch(rep):
    from . import configs
    from .learned import LearnedMC
    s = configs.c5_learned(seed=1)
    lm = LearnedMC([s] * 16, seed=3)
    bb = lm.bb
    bb.begin_sweep()
    x, y = bb.feature_buffers()
    for step in range(3 + rep):
        bb.propose(step, x)
        lm.net.forward(x, y)
        bb.decide(step, 1, y, bb.resid)
    torch.cuda.synchronize()
    bb.check_status()


def c4_hist(rep):
    from . import configs
    from .batch import BatchBoxes
    bb = BatchBoxes(configs.c4_batch(seed=1))
    for _ in range(3 + rep):
        bb.histograms()
    torch.cuda.synchronize()


CASES = {"c3_molfit": c3_molfit, "c3_atogen": c3_atogen, "c5_batch": c5_batch, "c4_hist": c4_hist}

if __name__ == "__main__":
    case = sys.argv[1]
    rep = int(sys.argv[2]) if len(sys.argv) > 2 else 1
    CASES[case](rep)
    print(f"{case}: ok")
