"""Long runs of the device iteration against the oracle's, across independent seeds.

Single-iteration bit-exactness does not show that a long run samples what the reference
samples: the fast summations, the device cosine and exponential, and the speculative resolve
can each shift a chain.  This test runs the EPSR iteration of the path (cell list, fmolec1,
5 molfit sweeps, atogen, gensq, ptgnsq's difference, press, fit_expansion, the EP refinement,
the running averages, stog) on configuration C1 (100 water) for 30 iterations from 8 ran1
seeds on the device -- fast sums, the mode the benchmark runs -- and from 8 other seeds on
the CPU oracle (the C restatement of the reference, one process per seed).  The first 10
iterations are dropped; per seed the remaining iterations are averaged, and for each
observable the two ensembles' means must agree within four standard errors:
  * the energy per molecule (press, ato_manipulation_rev4.py:4051);
  * the O-O partial g(r) histogram over the first peak (2.55-3.15 A, atogen :3640-3899) and
    over the first minimum (3.3-3.6 A);
  * the O-H and H-H partial S(Q) at Q = 2 A^-1 (gensq epsr_standalone_rev3.py:4731-4802);
  * the data-fit chi^2 of fit_expansion (:4806-4921)."""

import multiprocessing as mp

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

NIT, BURN, NSEED = 30, 10, 8


def _observables(wav, sofq, energy, chisq, b):
    ld = b.npt + 1
    w = np.asarray(wav, np.float64).reshape(2, b.npairs, ld)
    s = np.asarray(sofq, np.float64).reshape(2, b.npairs, -1)
    # pair 0 = O-O, 1 = O-H, 2 = H-H (type order O, H); r bin j at (j-2)*0.03 A
    peak = w[1, 0, 2 + 85:2 + 105].sum()
    trough = w[1, 0, 2 + 110:2 + 120].sum()
    return np.array([float(energy), peak, trough, s[1, 1, 40], s[1, 2, 40], float(np.sum(chisq))])


def _cpu_run(seed):
    from epsr_python_translation_b200 import configs
    from oracle.workload import CpuIteration
    wl = configs.make_workload("c1_water", ntimes=5)
    it = CpuIteration(wl, ran1_seed=seed)
    out = []
    for _ in range(NIT):
        it.step()
        out.append(_observables(it.wav, it.sofq, it.press["energy"], it.chisq, it.box))
    return np.array(out)


def test_device_long_runs_agree_with_oracle_across_seeds():
    from epsr_python_translation_b200 import configs
    from epsr_python_translation_b200.iteration import EpsrIteration
    ctx = mp.get_context("spawn")
    with ctx.Pool(NSEED) as pool:
        cpu_async = pool.map_async(_cpu_run, [-(101 + i) for i in range(NSEED)])
        wl = configs.make_workload("c1_water", ntimes=5)
        gpu = []
        for i in range(NSEED):
            it = EpsrIteration(wl, strict=False, ran1_seed=-(1 + i), native=False)
            out = []
            for _ in range(NIT):
                it.step()
                out.append(_observables(it.d.a_wav.cpu().numpy(), it.sofq.cpu().numpy(), it.energy, it.chisq,
                                        it.box))
            gpu.append(np.array(out))
        cpu = cpu_async.get(timeout=900)
    g = np.array([r[BURN:].mean(axis=0) for r in gpu])
    c = np.array([r[BURN:].mean(axis=0) for r in cpu])
    names = ["energy", "g(r) O-O peak", "g(r) O-O minimum", "S(Q) O-H", "S(Q) H-H", "chi^2"]
    for k, name in enumerate(names):
        se = np.sqrt(g[:, k].var(ddof=1) / NSEED + c[:, k].var(ddof=1) / NSEED)
        assert abs(g[:, k].mean() - c[:, k].mean()) <= 4 * se + 1e-9 * abs(c[:, k].mean()), \
            (name, g[:, k].mean(), c[:, k].mean(), se)
