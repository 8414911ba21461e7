"""The decision check used by the GPU chain tests can fail: mistakes planted in the oracle's
own trace (on the CPU) are caught, and only a decision at the threshold of its draw passes."""

import math

import numpy as np
import pytest

from epsr_python_translation_b200.box import BoxArrays, Ran1State
from oracle import oracle
from tests import goldens
from tests.chain_check import check_decisions

f32 = np.float32
RTOL = 1e-5


@pytest.fixture(scope="module")
def trace():
    z = goldens.load("c1_water")
    ob = BoxArrays.from_golden(z)
    oc = oracle.cell_list(ob, int(z["in_nmolcell"]), f32(z["in_sepmax"]))
    ost = oracle.fmolec1(ob, oc, z["in_eintra"])
    nmt = ob.nmoltype
    omc = dict(rejrate=f32(z["in_rejrate"]), stepr=f32(z["in_stepr"]), stepm=f32(z["in_stepm"]),
               wholerot=z["in_wholerot"].copy(), wholetrans=z["in_wholetrans"].copy(),
               internrot=np.zeros(nmt, f32), interntrans=np.zeros(nmt, f32), ireset=0)
    _, tr, _ = oracle.molfit(ob, oc, ost, omc, Ran1State.from_golden(z, "mf_ran1_before_"))
    return ob.simt, tr


def _interior_move(simt, tr):
    """A move whose exponent is inside (0, 20) and whose draw is far from its threshold."""
    for k in range(int(tr["nmoves"])):
        e = float(tr["den"][k]) / float(simt)
        thr = -float(simt) * math.log(float(tr["u"][k]))
        if 0.5 < e < 15 and abs(thr - tr["den64"][k]) > 100 * (RTOL * tr["scale64"][k] + 1e-6):
            return k
    raise AssertionError("no interior move in the trace")


def test_oracle_chain_passes_its_own_check(trace):
    simt, tr = trace
    assert check_decisions(tr["den"], tr["acc"], tr, simt, RTOL) == "same"


def test_flipped_decision_away_from_threshold_is_caught(trace):
    simt, tr = trace
    k = _interior_move(simt, tr)
    acc = tr["acc"].copy()
    acc[k] ^= 1
    with pytest.raises(AssertionError):
        check_decisions(tr["den"], acc, tr, simt, RTOL)


def test_energy_outside_tolerance_is_caught(trace):
    simt, tr = trace
    k = _interior_move(simt, tr)
    den = tr["den"].copy()
    den[k] = f32(den[k] + 10 * (RTOL * tr["scale64"][k] + 1e-6))
    with pytest.raises(AssertionError):
        check_decisions(den, tr["acc"], tr, simt, RTOL)


def test_decision_at_the_threshold_of_its_draw_may_part(trace):
    """Put the draw exactly at the threshold of the exact change: the two decisions are then
    both admissible, and the flipped one ends the comparison instead of failing it."""
    simt, tr = trace
    k = _interior_move(simt, tr)
    t = dict(tr)
    t["u"] = tr["u"].copy()
    t["u"][k] = f32(math.exp(-tr["den64"][k] / float(simt)))
    acc = tr["acc"].copy()
    acc[k] ^= 1
    den = tr["den"].copy()
    # the device's own change sits on the other side of the threshold, within tolerance
    tol = RTOL * tr["scale64"][k] + 1e-6
    den[k] = f32(tr["den64"][k] + (tol / 2 if acc[k] == 0 else -tol / 2))
    assert check_decisions(den, acc, t, simt, RTOL) == "parted"
