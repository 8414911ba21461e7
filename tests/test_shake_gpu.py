"""The intramolecular branch of molfit (molfit.py:124-174, then :465-536) and en_mole_intra
(:1327) on the device through the C ABI (epsr_molfit_shake, epsr_en_mole_intra), against the
reference run on seeded systems (tests/golden/shake.npz), bit for bit over two cycles; the
pair store the cycles start from is built by the device cell list and fmolec1 from the
reference's intramolecular energies."""

import numpy as np
import pytest
import torch

from epsr_python_translation_b200.box import BoxArrays, Ran1State, trsteps
from tests.goldens import GOLDEN, assert_bits_equal
from tests.test_shake_oracle import CASES, Prefixed

pytestmark = pytest.mark.gpu
f32 = np.float32


def _setup(name):
    from epsr_python_translation_b200.device import DeviceBox
    from epsr_python_translation_b200.intra import IntraModel
    z = np.load(GOLDEN + "/shake.npz")
    p = Prefixed(z, name + "_")
    box = BoxArrays.from_golden(p)
    d = DeviceBox(box)
    d.cell_list(10, box.sepmax)
    d.fmolec1(p["eintra"], strict=True)
    sc = p["scal"]
    tmax, tmin = trsteps(box.natomr)
    d.mc_setup(rejrate=0.75, stepr=1.0, stepm=1.0, wholerot=p["wholerot_in"], wholetrans=p["wholetrans_in"],
               internrot=p["internrot_in"], interntrans=p["interntrans_in"], ran1=Ran1State.from_golden(p, "ran1_before_"),
               trstepmax=tmax, trstepmin=tmin, fadds=p["fadds_in"])
    model = IntraModel(d, nbond=p["nbond"], iabond=p["iabond"], tbond=p["tbond"], amassa=p["amassa"],
                       amassr=p["amassr"], xav=p["xav"], xav1=p["xav1"], stepcl=sc[0], sizefactor=sc[1], tempb=sc[2],
                       tempang=sc[3], simt=sc[4], refine_intra=bool(sc[5]), refine_intra_fac=sc[6])
    return p, box, d, model, f32(sc[7])


@pytest.mark.parametrize("name", CASES)
def test_en_mole_intra_device_matches_reference(name):
    p, box, d, model, _ = _setup(name)
    assert_bits_equal(model.en_mole_intra().cpu().numpy(), p["eintra"], f"{name} eintra")


@pytest.mark.parametrize("name", CASES)
def test_shake_cycle_device_matches_reference(name):
    p, box, d, model, stepmi = _setup(name)
    co = d.download_coords()
    for k in co:                                    # the cycles start where the reference's did
        assert_bits_equal(co[k], p["in_" + k], f"{name} start {k}")
    st = d.download_store()
    assert_bits_equal(st["ergpair"], p["in_ergpair"], f"{name} start store")
    faddbs = torch.tensor([float(p["faddbs_in"])], dtype=torch.float32, device="cuda")
    for c in range(int(p["cycles"])):
        q = f"c{c}_"
        nmovei = model.molfit_shake(stepmi, faddbs).cpu().numpy()
        co = d.download_coords()
        for k in co:
            assert_bits_equal(co[k], p[q + k], f"{name} cycle {c} {k}")
        assert_bits_equal(d.download_store()["ergpair"], p[q + "ergpair"], f"{name} cycle {c} ergpair")
        mc = d.download_mc()
        for k in ("interntrans", "internrot", "wholerot", "wholetrans"):
            assert_bits_equal(mc[k], p[q + k], f"{name} cycle {c} {k}")
        assert np.array_equal(nmovei, p[q + "nmovei"].reshape(-1)), (nmovei, p[q + "nmovei"])
        assert np.array_equal(mc["nwhole"], p[q + "nwhole"]) and np.array_equal(mc["nmovem"], p[q + "nmovem"])
        assert_bits_equal(np.array([mc["fadds"], faddbs.cpu().numpy()[0]], f32),
                          np.array([p[q + "fadds"], p[q + "faddbs"]], f32), f"{name} cycle {c} fadds, faddbs")
        r = mc["ran1"]
        assert (r.idum, r.iy) == (int(p[q + "ran1_after_idum"]), int(p[q + "ran1_after_iy"]))
        assert np.array_equal(r.iv, p[q + "ran1_after_iv"])


def test_shake_refuses_rotational_groups_before_any_change():
    from epsr_python_translation_b200._lib import EpsrGpuError
    from epsr_python_translation_b200.intra import IntraModel
    p, box, d, model, stepmi = _setup("mix")
    ngrot = np.zeros(box.nmol, np.int32)
    ngrot[3] = 1
    m2 = IntraModel(d, nbond=p["nbond"], iabond=p["iabond"], tbond=p["tbond"], amassa=p["amassa"], amassr=p["amassr"],
                    xav=p["xav"], xav1=p["xav1"], stepcl=p["scal"][0], simt=p["scal"][4], ngrot=ngrot)
    before = d.download_coords()
    r0 = d.m_ran1.cpu().numpy().copy()
    with pytest.raises(EpsrGpuError):
        m2.molfit_shake(stepmi, torch.zeros(1, device="cuda"))
    after = d.download_coords()
    for k in before:
        assert_bits_equal(after[k], before[k], k)
    assert np.array_equal(d.m_ran1.cpu().numpy(), r0)
