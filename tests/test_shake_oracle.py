"""The C restatement of the intramolecular branch of molfit (molfit.py:124-174, the cycle
taken when nisum >= intra, with the step adaptation :465-536) and of en_mole_intra (:1327)
against the reference run on seeded systems (tests/golden/shake.npz, made by
tests/golden/make_golden_shake.py), bit for bit over two cycles: coordinates, stored energies,
step sizes, counts, fadds/faddbs and the ran1 stream."""

import numpy as np
import pytest

from epsr_python_translation_b200.box import BoxArrays, Ran1State
from oracle import oracle
from tests.goldens import GOLDEN, assert_bits_equal

f32 = np.float32
CASES = ["mix", "water"]


class Prefixed:
    def __init__(self, z, p):
        self.z, self.p = z, p

    def __getitem__(self, k):
        return self.z[self.p + k]

    def __contains__(self, k):
        return self.p + k in self.z.files


def case(z, name):
    p = Prefixed(z, name + "_")
    box = BoxArrays.from_golden(p)
    for k in ("xa", "ya", "za", "xadd", "yadd", "zadd"):
        getattr(box, k)[:] = p["in_" + k]
    sc = p["scal"]
    model = dict(nbond=p["nbond"], iabond=p["iabond"], tbond=p["tbond"], amassa=p["amassa"], amassr=p["amassr"],
                 xav=p["xav"], xav1=p["xav1"], stepcl=sc[0], sizefactor=sc[1], tempb=sc[2], tempang=sc[3], simt=sc[4],
                 refine_intra=bool(sc[5]), refine_intra_fac=sc[6])
    M = int(p["in_nnbrefmax"])
    n = int(p["in_nergpair"])
    st = dict(nnbrefmax=M, nergpair=n, nergpairm=np.ascontiguousarray(p["in_nergpairm"], np.int32),
              molergpair=np.ascontiguousarray(p["in_molergpair"][:M].T - 1, np.int32).reshape(-1),
              ergpairref=np.ascontiguousarray(p["in_ergpairref"][:M].T, np.int32).reshape(-1),
              ergpair=np.array(p["in_ergpair"][:n], f32))
    mc = dict(rejrate=f32(0.75), ireset=0, **{k: np.array(p[k + "_in"], f32) for k in
                                              ("wholerot", "wholetrans", "internrot", "interntrans")})
    return p, box, model, st, mc, f32(sc[7])


@pytest.mark.parametrize("name", CASES)
def test_en_mole_intra_oracle_matches_reference(name):
    z = np.load(GOLDEN + "/shake.npz")
    p, box, model, _, _, _ = case(z, name)
    assert_bits_equal(oracle.en_mole_intra_all(box, model), p["eintra"], f"{name} eintra")


@pytest.mark.parametrize("name", CASES)
def test_shake_cycle_oracle_matches_reference(name):
    z = np.load(GOLDEN + "/shake.npz")
    p, box, model, st, mc, stepmi = case(z, name)
    ran1 = Ran1State.from_golden(p, "ran1_before_")
    fadds, faddbs, eo = f32(p["fadds_in"]), f32(p["faddbs_in"]), f32(p["ergold1_in"])
    for c in range(int(p["cycles"])):
        q = f"c{c}_"
        fadds, faddbs, nmovei, eo, ran1 = oracle.molfit_shake(box, st, mc, model, stepmi, ran1, fadds, faddbs, eo)
        for k in ("xa", "ya", "za", "xadd", "yadd", "zadd"):
            assert_bits_equal(getattr(box, k), p[q + k], f"{name} cycle {c} {k}")
        assert_bits_equal(st["ergpair"], p[q + "ergpair"], f"{name} cycle {c} ergpair")
        for k in ("interntrans", "internrot", "wholerot", "wholetrans"):
            assert_bits_equal(mc[k], p[q + k], f"{name} cycle {c} {k}")
        assert np.array_equal(nmovei, p[q + "nmovei"].reshape(-1)), (nmovei, p[q + "nmovei"])
        assert_bits_equal(np.array([fadds, faddbs], f32), np.array([p[q + "fadds"], p[q + "faddbs"]], f32),
                          f"{name} cycle {c} fadds, faddbs")
        assert (ran1.idum, ran1.iy, ran1.mcall) == (int(p[q + "ran1_after_idum"]), int(p[q + "ran1_after_iy"]),
                                                     int(p[q + "ran1_after_mcall"]))


def test_shake_golden_exercises_the_first_slot_rule():
    """Water molecule 0 has an intramolecular energy of exactly 0, so its first stored energy
    is an intermolecular pair -- the case the ordered pass exists for -- and the mixture
    case has rejected moves."""
    z = np.load(GOLDEN + "/shake.npz")
    assert z["water_eintra"][0] == 0.0
    assert z["mix_c0_nmovei"][1].sum() > 0
