"""The fast fit's summation against the reference's, statistically, on the CPU.

The device's fast fit mode (the one the iteration driver and the benchmark run) sums each
trial's chi^2 in double and rounds it once to float32, where fit_expansion
(epsr_standalone_rev3.py:4806-4921) sums it sequentially in float32.  The device matches the
oracle's restatement of the fast summation bit for bit (tests/test_gpu_parity.py); this file
shows on the oracle alone that the two summations give chains with the same outcome: over
16 seeded C2-size fits (600 Q rows x 116 terms), the paired differences of log final chi^2,
of the final rejection ratio and of log step size have means within three standard errors of
zero, and the fitted curves agree to the fit's own resolution."""

import numpy as np

from epsr_python_translation_b200 import configs
from epsr_python_translation_b200.box import Ran1State
from oracle import oracle

f32 = np.float32


def _fit(seed, fast):
    nq, nt = 600, 116
    q = configs.qgrid(nq, 0.05)
    expr = configs.ep_basis(q, nt)
    rng = np.random.default_rng(seed)
    yin = np.zeros(nq + 1, f32)
    yin[1:] = (rng.standard_normal(nq) * 0.05 + 0.2 * np.sin(q[1:] * (1 + seed % 3))).astype(f32)
    wtold = np.zeros(nt + 1, f32)
    wtold[1:] = (rng.standard_normal(nt) * 0.01).astype(f32)
    ref, _ = oracle.fit_expansion(yin, expr, wtold, f32(0.01), 1, nq, 1, nt, 1000, 10, Ran1State(idum=-seed),
                                  fast=fast)
    return ref, yin


def _within(d, what):
    d = np.asarray(d, np.float64)
    m, se = d.mean(), d.std(ddof=1) / np.sqrt(d.size)
    assert abs(m) <= 3 * se + 1e-12, (what, m, se)


def test_fast_and_reference_summation_fit_alike():
    seeds = range(101, 117)
    dchi, drej, dstep, parted = [], [], [], 0
    for s in seeds:
        a, yin = _fit(s, False)
        b, _ = _fit(s, True)
        parted += int(not np.array_equal(a["wt"], b["wt"]))
        dchi.append(np.log(float(b["chisq"])) - np.log(float(a["chisq"])))
        drej.append(float(b["rejrat"]) - float(a["rejrat"]))
        dstep.append(np.log(float(b["stepr"])) - np.log(float(a["stepr"])))
        # both fits reproduce the data to the same resolution (relative chi^2 within 20%)
        assert abs(dchi[-1]) < 0.2, (s, a["chisq"], b["chisq"])
    assert parted > 0   # the summations do differ, so the comparison is not vacuous
    _within(dchi, "log chi^2")
    _within(drej, "rejection ratio")
    _within(dstep, "log step")
