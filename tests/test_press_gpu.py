"""press on the device (epsr_press) against the reference's press on the golden systems:
strict summation bit for bit (energy and pressure); the fast summation (double, parallel)
within 1e-6 relative of the oracle's double sums of the same float32 pair terms (the
reference's float32 sequential sum itself differs from those by up to ~1e-5 at C2 size)."""

import numpy as np
import pytest

from epsr_python_translation_b200.box import BoxArrays
from epsr_python_translation_b200.device import press_scalars
from tests import goldens
from tests.goldens import assert_bits_equal
from tests.test_press_oracle import CASES, press_case

pytestmark = pytest.mark.gpu
f32 = np.float32


def _device_store(case):
    from epsr_python_translation_b200.device import DeviceBox
    z = goldens.load(case)
    box = BoxArrays.from_golden(z)
    d = DeviceBox(box)
    d.cell_list(int(z["in_nmolcell"]), f32(z["in_sepmax"]))
    d.fmolec1(z["in_eintra"], strict=True)
    return z, box, d


@pytest.mark.parametrize("case", CASES)
def test_press_device_matches_reference(case):
    p = press_case(case)
    z, box, d = _device_store(case)
    assert d.download_store()["nergpair"] == int(p[case + "_nergpair"])
    sumc, presst = d.press(strict=True)
    energy, pressc = press_scalars(box.nmol, sumc, presst, p[case + "_simt"], p[case + "_volume"])
    assert_bits_equal(energy, p[case + "_energy"], "energy")
    assert_bits_equal(pressc, p[case + "_pressc"], "pressc")
    # the fast summation against the oracle's double sums of the same terms
    from oracle import oracle
    ob = BoxArrays.from_golden(z)
    oc = oracle.cell_list(ob, int(z["in_nmolcell"]), f32(z["in_sepmax"]))
    ref = oracle.press(ob, oracle.fmolec1(ob, oc, z["in_eintra"]), box.npt1, p[case + "_simt"], p[case + "_volume"])
    s2, p2 = d.press(strict=False)
    assert abs(float(s2) - ref["sum64"]) <= 1e-6 * abs(ref["sum64"]) + 1e-6
    assert abs(p2 - ref["presst"]) <= 1e-9 * abs(ref["presst"]) + 1e-9
