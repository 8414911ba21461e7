"""The pair path on a triclinic cell (minimagec.py:13-45 through fractional coordinates) against
the C oracle, whose triclinic minimum image is pinned to the reference's own results
(tests/golden/triclinic.npz): a golden water box with its cell sheared (b and c leaning on a),
through the cell list, the pair store, the sequential molfit cycle and the fast cycle (whose
energy pass takes the division form of the table index there, the bin-edge form being for cubic
boxes only), with the oracle's cosines injected.
"""

import numpy as np
import pytest

from epsr_python_translation_b200.box import BoxArrays, Ran1State, trsteps
from oracle import oracle
from tests import goldens
from tests.chain_check import check_decisions
from tests.goldens import assert_bits_equal

pytestmark = pytest.mark.gpu
f32 = np.float32

ENERGY_RTOL = 1e-5   # relative to the sum of |pair energies| of the move

# alatx, blatx, clatx, blaty, claty, clatz (box units) and the cell vectors a, b, c
LAT6 = np.array([1.0, 0.1, 0.05, 0.995, 0.08, 0.99], f32)
LAT9 = np.array([1.0, 0.0, 0.0, 0.1, 0.995, 0.0, 0.05, 0.08, 0.99], f32)


def _box(z):
    box = BoxArrays.from_golden(z)
    box.cubic = False
    box.lat6 = LAT6.copy()
    box.lat9 = LAT9.copy()
    return box


def _mc_args(z, box):
    nmt = box.nmoltype
    return dict(rejrate=f32(z["in_rejrate"]), stepr=f32(z["in_stepr"]), stepm=f32(z["in_stepm"]),
                wholerot=z["in_wholerot"].copy(), wholetrans=z["in_wholetrans"].copy(),
                internrot=np.zeros(nmt, f32), interntrans=np.zeros(nmt, f32))


@pytest.mark.parametrize("strict", [True, False])
def test_triclinic_store_and_cycle_match_oracle(strict):
    from epsr_python_translation_b200.device import DeviceBox
    z = goldens.load("c1_water")
    ob = _box(z)
    oc = oracle.cell_list(ob, int(z["in_nmolcell"]), f32(z["in_sepmax"]))
    ost = oracle.fmolec1(ob, oc, z["in_eintra"])
    d = DeviceBox(_box(z))
    d.cell_list(int(z["in_nmolcell"]), f32(z["in_sepmax"]))
    d.fmolec1(z["in_eintra"], strict=True)
    st = d.download_store()
    assert st["nergpair"] == ost["nergpair"]
    assert_bits_equal(st["ergpair"], ost["ergpair"][: ost["nergpair"]], "ergpair (triclinic)")
    args = _mc_args(z, ob)
    tmax, tmin = trsteps(ob.natomr)
    ran1 = Ran1State.from_golden(z, "mf_ran1_before_")
    d.mc_setup(ran1=ran1, trstepmax=tmax, trstepmin=tmin, **{k: v.copy() if hasattr(v, "copy") else v
                                                             for k, v in args.items()})
    omc = dict(args, ireset=0)
    for cyc in range(2):
        _, tr, ran1 = oracle.molfit(ob, oc, ost, omc, ran1)
        d.molfit(strict=strict, cos_override=tr["cosv"])
        d.check_status()
        m = d.download_mc()
        co = d.download_coords()
        if strict:
            assert np.array_equal(m["acc"], tr["acc"]), cyc
        elif check_decisions(m["den"], m["acc"], tr, ob.simt, ENERGY_RTOL) == "parted":
            return
        for k in ("xa", "ya", "za", "xadd", "yadd", "zadd"):
            assert_bits_equal(co[k], getattr(ob, k), f"cycle {cyc} {k}")
        assert_bits_equal(d.download_store()["ergpair"], ost["ergpair"][: ost["nergpair"]], f"cycle {cyc} ergpair")
        assert m["ran1"].idum == ran1.idum and np.array_equal(m["ran1"].iv, ran1.iv)
