"""Internal rotations of rotational groups in the device's whole-molecule cycle (molfit.py:
295-360, rotati :589, en_change_intra :763) and in its intramolecular cycle (:124-267) against
the reference run on a 20 DMSO + 40 water box whose methyl groups are ROT groups
(tests/golden/rot.npz, shake_rot.npz), with the reference's cosines injected: coordinates, stored energies (including the first-slot rule after a rejected rotation
followed by an accepted move), step sizes, ninter/nwhole/nmovem, fadds/faddbs and the ran1
state bit for bit over two cycles."""

import numpy as np
import pytest

from epsr_python_translation_b200.box import Ran1State, trsteps
from tests.goldens import assert_bits_equal
from tests.test_rot_oracle import load

pytestmark = pytest.mark.gpu
f32 = np.float32


@pytest.mark.parametrize("name", ["rot.npz", "dih_rot.npz"])
def test_rotation_cycles_device_match_reference(name):
    from epsr_python_translation_b200.device import DeviceBox
    from epsr_python_translation_b200.intra import IntraModel
    z, box, st, mc, rot = load(name)
    d = DeviceBox(box)
    d.cell_list(int(z["in_nmolcell"]), f32(z["in_sepmax"]))
    d.fmolec1(z["eintra"], strict=True)
    s0 = d.download_store()
    assert_bits_equal(s0["ergpair"], st["ergpair"], "store before the cycles")
    tmax, tmin = trsteps(box.natomr)
    d.mc_setup(rejrate=f32(0.75), stepr=f32(z["in_stepr"]), stepm=f32(z["in_stepm"]), wholerot=z["wholerot_in"],
               wholetrans=z["wholetrans_in"], internrot=z["internrot_in"], ran1=Ran1State.from_golden(z, "ran1_before_"),
               trstepmax=tmax, trstepmin=tmin, fadds=f32(z["fadds_in"]))
    model = dict(rot["model"])
    im = IntraModel(d, **model)
    if name == "dih_rot.npz":
        # the stored intramolecular energies with the dihedral term, on the device
        assert_bits_equal(im.en_mole_intra().cpu().numpy(), z["eintra"], "eintra with dihedrals")
    d.set_rotations(im, z["rot_nrf"], z["rot_nrl"], z["rot_axis"], z["rot_first"], z["rot_last"], z["rot_atoms"],
                    stepri=1.0, faddbs=f32(z["faddbs_in"]))
    for c in range(int(z["cycles"])):
        q = f"c{c}_"
        d.molfit(strict=True, cos_override=z[q + "cos"], rotcycle=True)
        d.check_status()
        m = d.download_mc()
        co = d.download_coords()
        for k in ("xa", "ya", "za", "xadd", "yadd", "zadd"):
            assert_bits_equal(co[k], z[q + k], f"cycle {c} {k}")
        assert_bits_equal(d.download_store()["ergpair"], z[q + "ergpair"], f"cycle {c} ergpair")
        for k in ("internrot", "wholerot", "wholetrans"):
            assert_bits_equal(m[k], z[q + k], f"cycle {c} {k}")
        assert np.array_equal(d.m_ninter.cpu().numpy(), z[q + "ninter"].reshape(-1))
        assert np.array_equal(m["nwhole"].reshape(-1), z[q + "nwhole"].reshape(-1))
        assert np.array_equal(m["nmovem"].reshape(-1), z[q + "nmovem"].reshape(-1))
        assert_bits_equal(np.array([m["fadds"], d.m_faddbs.cpu().numpy()[0]], f32),
                          np.array([z[q + "fadds"], z[q + "faddbs"]], f32), f"cycle {c} fadds, faddbs")
        assert m["ran1"].idum == int(z[q + "ran1_after_idum"])
        assert np.array_equal(m["ran1"].iv, z[q + "ran1_after_iv"])


@pytest.mark.parametrize("name", ["rot.npz", "dih_rot.npz"])
def test_rotation_dropin_matches_reference(name):
    """PairPath.molfit on COMMON stand-ins that carry the reference's rotational groups
    (molecom_mod labaxi/rotf/rotl/labrot, clustercom ngrot/nrf/nrl, of type ROT or DIH with
    their dihedral angles) and intramolecular model: the whole-molecule cycles with internal
    rotations run on the device and leave the COMMON state equal to the reference's; no host
    routine ran."""
    _rotation_dropin(name, shake=False)


@pytest.mark.parametrize("name", ["shake_rot.npz", "dih_shake.npz"])
def test_shake_rotation_dropin_matches_reference(name):
    """As above for the intramolecular cycles (nisum >= intra) of the same box: atom moves and
    internal rotations on the device, the COMMON state (nmovei, ninter, nstepreject and
    interntrans included) equal to the reference's; no host routine ran."""
    _rotation_dropin(name, shake=True)


def _rotation_dropin(name, shake):
    from epsr_python_translation_b200 import dropin
    from tests import fake_common
    z, c, mods, calls = fake_common.common_with_groups(name, shake)
    mc, cc, erd, r = c.molecom, c.clustercom, c.ergpairreference, c.ran1com
    nmol, nmt = cc.nmol, int(cc.nmoltype)
    path = dropin.PairPath(c, mods, strict=True)
    path.install(dropin.ROUTINES)
    mods["cellneighbourlist"].initialise_cellneighbourlist(int(z["in_nmolcell"]), cc.xadd, cc.yadd, cc.zadd, nmol,
                                                          f32(z["in_sepmax"]))
    mods["ato_manipulation_rev4"].fmolec1(0, 0, f32(0), f32(0), f32(0), f32(0))
    assert_bits_equal(erd.ergpair[1:erd.nergpair + 1], z["in_ergpair"], "store before the cycles")
    fake_common.set_ran1(c, z, "ran1_before_")
    fadds, faddbs = f32(z["fadds_in"]), f32(z["faddbs_in"])
    nisum = 1
    for cyc in range(int(z["cycles"])):
        q = f"c{cyc}_"
        path.cos_override = z[q + "cos"]
        if shake:
            fadds, faddbs, nisum = mods["molfit"].molfit(fadds, faddbs, 1, 1, 5, 0)
        else:
            fadds, faddbs, nisum = mods["molfit"].molfit(fadds, faddbs, nisum, 100, 1, 0)
        assert nisum == int(z[q + "nisum"])
        assert_bits_equal(np.array([fadds, faddbs], f32), np.array([z[q + "fadds"], z[q + "faddbs"]], f32),
                          q + "fadds, faddbs")
        for k, arr in (("xa", mc.xa), ("ya", mc.ya), ("za", mc.za), ("xadd", cc.xadd), ("yadd", cc.yadd),
                       ("zadd", cc.zadd)):
            assert_bits_equal(arr[1:], z[q + k], q + k)
        assert_bits_equal(erd.ergpair[1:erd.nergpair + 1], z[q + "ergpair"], q + "ergpair")
        for k in ("internrot", "wholerot", "wholetrans") + (("interntrans",) if shake else ()):
            assert_bits_equal(getattr(cc, k)[1:], z[q + k], q + k)
        for k in ("ninter", "nwhole", "nmovem") + (("nmovei",) if shake else ()):
            assert np.array_equal(getattr(cc, k)[1:3, 1:nmt + 1], z[q + k]), k
        if shake:
            assert np.array_equal(cc.nstepreject[1:], z[q + "nstepreject"])
        assert (r.idum, r.iy, r.mcall) == (int(z[q + "ran1_after_idum"]), int(z[q + "ran1_after_iy"]),
                                           int(z[q + "ran1_after_mcall"]))
    assert not [k for k in calls if k.startswith("host:")], calls


@pytest.mark.parametrize("name", ["shake_rot.npz", "dih_shake.npz"])
def test_shake_rotation_cycles_device_match_reference(name):
    """molfit's intramolecular cycle on a box with ROT groups (molfit.py:124-267: each
    molecule's atom moves, then its methyl groups rotated and tested with the intermolecular
    change, molecules in index order) through epsr_molfit_shake with the reference's cosines
    injected: coordinates, stored energies, step sizes, nmovei/ninter, nstepreject, fadds/faddbs
    and the ran1 state equal the reference's bit for bit over two cycles
    (tests/golden/shake_rot.npz)."""
    import torch

    from epsr_python_translation_b200.device import DeviceBox
    from epsr_python_translation_b200.intra import IntraModel
    from tests.test_rot_oracle import load_shake
    z, box, st, mc, rot = load_shake(name)
    d = DeviceBox(box)
    d.cell_list(int(z["in_nmolcell"]), f32(z["in_sepmax"]))
    d.fmolec1(z["eintra"], strict=True)
    assert_bits_equal(d.download_store()["ergpair"], st["ergpair"], "store before the cycles")
    tmax, tmin = trsteps(box.natomr)
    d.mc_setup(rejrate=f32(0.75), stepr=f32(z["in_stepr"]), stepm=f32(z["in_stepm"]), wholerot=z["wholerot_in"],
               wholetrans=z["wholetrans_in"], internrot=z["internrot_in"], interntrans=z["interntrans_in"],
               ran1=Ran1State.from_golden(z, "ran1_before_"), trstepmax=tmax, trstepmin=tmin, fadds=f32(z["fadds_in"]))
    im = IntraModel(d, **dict(rot["model"]))
    d.set_rotations(im, z["rot_nrf"], z["rot_nrl"], z["rot_axis"], z["rot_first"], z["rot_last"], z["rot_atoms"],
                    stepri=1.0)
    fb = torch.tensor([float(z["faddbs_in"])], dtype=torch.float32, device=d.dev)
    for c in range(int(z["cycles"])):
        q = f"c{c}_"
        d.set_cos_override(z[q + "cos"])
        nmovei = im.molfit_shake(f32(z["stepmi"]), fb).cpu().numpy()
        d.check_status()
        m = d.download_mc()
        co = d.download_coords()
        for k in ("xa", "ya", "za", "xadd", "yadd", "zadd"):
            assert_bits_equal(co[k], z[q + k], f"cycle {c} {k}")
        assert_bits_equal(d.download_store()["ergpair"], z[q + "ergpair"], f"cycle {c} ergpair")
        for k in ("interntrans", "internrot", "wholerot", "wholetrans"):
            assert_bits_equal(m[k], z[q + k], f"cycle {c} {k}")
        assert np.array_equal(nmovei, z[q + "nmovei"].reshape(-1))
        assert np.array_equal(d.m_ninter.cpu().numpy(), z[q + "ninter"].reshape(-1))
        assert np.array_equal(m["nstepreject"], z[q + "nstepreject"])
        assert_bits_equal(np.array([m["fadds"], fb.cpu().numpy()[0]], f32),
                          np.array([z[q + "fadds"], z[q + "faddbs"]], f32), f"cycle {c} fadds, faddbs")
        assert m["ran1"].idum == int(z[q + "ran1_after_idum"])
        assert np.array_equal(m["ran1"].iv, z[q + "ran1_after_iv"])
