"""press (ato_manipulation_rev4.py:3903-4062): the C restatement against the reference run
on the golden systems (tests/golden/press.npz, made by make_golden_press.py): energy and
pressure bit for bit, and the per-file rescaling."""

import os

import numpy as np
import pytest

from epsr_python_translation_b200.box import BoxArrays
from oracle import oracle
from tests import goldens
from tests.goldens import assert_bits_equal

f32 = np.float32
PRESS = os.path.join(goldens.GOLDEN, "press.npz")
CASES = ["c1_water", "mix_small", "silica", "c2_mixture"]


def press_case(case):
    p = np.load(PRESS)
    if case + "_energy" not in p.files:
        pytest.skip(f"no press golden for {case}")
    return p


def oracle_store(z, box):
    oc = oracle.cell_list(box, int(z["in_nmolcell"]), f32(z["in_sepmax"]))
    return oracle.fmolec1(box, oc, z["in_eintra"])


@pytest.mark.parametrize("case", CASES)
def test_press_oracle_matches_reference(case):
    p = press_case(case)
    z = goldens.load(case)
    box = BoxArrays.from_golden(z)
    st = oracle_store(z, box)
    assert st["nergpair"] == int(p[case + "_nergpair"])
    r = oracle.press(box, st, box.npt1, p[case + "_simt"], p[case + "_volume"])
    assert_bits_equal(r["energy"], p[case + "_energy"], "energy")
    assert_bits_equal(r["pressc"], p[case + "_pressc"], "pressc")


@pytest.mark.parametrize("case", ["c1_water", "mix_small"])
def test_press_file_terms_match_reference(case):
    p = press_case(case)
    nmol = goldens.load(case)["sys_naf"].shape[0]
    ef, pf = oracle.press_file_terms(nmol, p[case + "_energf_in"], p[case + "_pressf_in"], f32(1.0),
                                     p[case + "_volume"])
    assert_bits_equal(ef, p[case + "_energf"], "energf")
    assert_bits_equal(pf, p[case + "_pressf"], "pressf")
