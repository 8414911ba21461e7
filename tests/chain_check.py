"""Decision check of a Monte Carlo chain against the oracle's trace of the same cycle.

A device chain that uses its own cosines proposes moves a rounding away from the
reference's, so its energy changes differ from the oracle's within the energy tolerance and
its decisions may differ where a draw falls between the two.  ``check_decisions`` accepts
exactly that and nothing else:
  * every energy change is within ``rtol`` x (sum of |pair energies| of the move) of the
    oracle's FP64 change;
  * every decision is the Metropolis rule (molfit.py:401-408) applied to the device's own
    energy change and the draw of the shared ran1 stream (unless the draw sits on the
    exponential itself);
  * a decision differs from the oracle's only where the threshold of that draw,
    -simt*ln(u), lies within the tolerance of the exact change; the chains part there.
"""

import math

import numpy as np

f32 = np.float32


def metropolis_accepts(den, temp, u):
    """molfit.py:401-408 for one move: ediff = (den + 0) * temp in float32; accept iff
    u < etest (10 when ediff <= 0, exp(-ediff) below 20, else 0), the exponential in double
    rounded once to float32 as the device evaluates it.  Returns (accept, etest)."""
    ediff = f32(f32(f32(den) + f32(0.0)) * f32(temp))
    if ediff <= 0:
        return True, f32(10.0)
    if ediff < 20:
        et = f32(np.exp(-np.float64(ediff)))
        return bool(f32(u) < et), et
    return False, f32(0.0)


def check_decisions(den, acc, tr, simt, rtol):
    """Raise AssertionError on a decision the tolerance does not allow.  Returns "parted"
    when the chains part at an allowed mismatch, else "same"."""
    temp = f32(1.0) / f32(simt)
    for k in range(int(tr["nmoves"])):
        tol = rtol * tr["scale64"][k] + 1e-6
        assert abs(float(den[k]) - tr["den64"][k]) <= tol, ("energy", k, den[k], tr["den64"][k], tol)
        u = float(tr["u"][k])
        own, et = metropolis_accepts(den[k], temp, u)
        if abs(u - float(et)) > 1e-6 * max(float(et), 1e-30):
            assert bool(acc[k]) == own, ("decision differs from the rule on its own energy change", k)
        if bool(acc[k]) != bool(tr["acc"][k]):
            thr = -float(simt) * math.log(u) if u > 0 else math.inf
            thr = min(thr, 20.0 * float(simt))
            assert abs(tr["den64"][k] - thr) <= tol, ("decision differs away from the threshold", k,
                                                      tr["den64"][k], thr, tol)
            return "parted"
    return "same"
