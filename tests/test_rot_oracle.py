"""The C restatement of molfit's whole-molecule cycle with internal rotations of rotational
groups (molfit.py:295-360, rotati :589, en_change_intra :763) against the reference run on a
20 DMSO + 40 water box with the methyl groups as ROT groups (tests/golden/rot.npz, made by
tests/golden/make_golden_rot.py), bit for bit over two cycles: coordinates, stored energies,
step sizes, ninter/nwhole/nmovem, fadds/faddbs and the ran1 stream."""

import numpy as np
import pytest

from epsr_python_translation_b200.box import BoxArrays, Ran1State
from oracle import oracle
from tests.goldens import GOLDEN, assert_bits_equal

f32 = np.float32


def _dih(z):
    """The golden's dihedral angles as the intramolecular model takes them, or None."""
    if "dih_cos" not in z.files:
        return None
    return dict(grp_nrf=z["rot_nrf"], grp_nrl=z["rot_nrl"], grp_axis=z["rot_axis"], grp_dih0=z["dih_grp0"],
                grp_isdih=z["dih_isdih"], dih_atoms=z["dih_atoms"], dih_cos=z["dih_cos"], dih_sin=z["dih_sin"],
                tempdih=z["tempdih"])


def load(name="rot.npz"):
    z = np.load(GOLDEN + "/" + name)
    box = BoxArrays.from_golden(z)
    for k in ("xa", "ya", "za", "xadd", "yadd", "zadd"):
        getattr(box, k)[:] = z["in_" + k]
    sc = z["scal"]
    model = dict(nbond=z["nbond"], iabond=z["iabond"], tbond=z["tbond"], amassa=z["amassa"], amassr=z["amassr"],
                 xav=z["xav"], xav1=z["xav1"], stepcl=sc[0], sizefactor=sc[1], tempb=sc[2], tempang=sc[3], simt=sc[4],
                 refine_intra=False, refine_intra_fac=f32(0.0), ngrot=z["ngrot"], dih=_dih(z))
    M = int(z["in_nnbrefmax"])
    n = int(z["in_nergpair"])
    st = dict(nnbrefmax=M, nergpair=n, nergpairm=np.ascontiguousarray(z["in_nergpairm"], np.int32),
              molergpair=np.ascontiguousarray(z["in_molergpair"][:M].T - 1, np.int32).reshape(-1),
              ergpairref=np.ascontiguousarray(z["in_ergpairref"][:M].T, np.int32).reshape(-1),
              ergpair=np.array(z["in_ergpair"][:n], f32))
    nmt = box.nmoltype
    mc = dict(rejrate=f32(0.75), stepr=f32(z["in_stepr"]), stepm=f32(z["in_stepm"]), ireset=0,
              wholerot=np.array(z["wholerot_in"], f32), wholetrans=np.array(z["wholetrans_in"], f32),
              internrot=np.array(z["internrot_in"], f32), interntrans=np.zeros(nmt, f32),
              ngrot=np.array(z["ngrot"], np.int32))
    rot = dict(model=model, nrf=z["rot_nrf"], nrl=z["rot_nrl"], axis=z["rot_axis"].reshape(-1), first=z["rot_first"],
               last=z["rot_last"], atoms=z["rot_atoms"], stepri=f32(1.0), rotcycle=1, faddbs=f32(z["faddbs_in"]))
    return z, box, st, mc, rot


@pytest.mark.parametrize("name", ["rot.npz", "dih_rot.npz"])
def test_rotation_golden_exercises_both_outcomes(name):
    z = np.load(GOLDEN + "/" + name)
    for c in range(int(z["cycles"])):
        ni = z[f"c{c}_ninter"]
        assert ni[0, 0] > 0 and 0 < ni[1, 0] < ni[0, 0]       # DMSO rotations tried, some rejected


@pytest.mark.parametrize("name", ["rot.npz", "dih_rot.npz"])
def test_rotation_cycles_oracle_matches_reference(name):
    z, box, st, mc, rot = load(name)
    if name == "dih_rot.npz":
        # the stored intramolecular energies include the dihedral term (en_mole_intra :1345)
        assert_bits_equal(oracle.en_mole_intra_all(box, rot["model"]), z["eintra"], "eintra with dihedrals")
    cells = oracle.cell_list(box, int(z["in_nmolcell"]), f32(z["in_sepmax"]))
    ran1 = Ran1State.from_golden(z, "ran1_before_")
    fadds = f32(z["fadds_in"])
    for c in range(int(z["cycles"])):
        q = f"c{c}_"
        fadds, tr, ran1 = oracle.molfit(box, cells, st, mc, ran1, fadds, rot=rot)
        rot["faddbs"] = tr["faddbs"]
        assert_bits_equal(tr["cosv"][: z[q + "cos"].size], z[q + "cos"], f"cycle {c} cos")
        for k in ("xa", "ya", "za", "xadd", "yadd", "zadd"):
            assert_bits_equal(getattr(box, k), z[q + k], f"cycle {c} {k}")
        assert_bits_equal(st["ergpair"], z[q + "ergpair"], f"cycle {c} ergpair")
        for k in ("internrot", "wholerot", "wholetrans"):
            assert_bits_equal(mc[k], z[q + k], f"cycle {c} {k}")
        assert np.array_equal(tr["ninter"], z[q + "ninter"].reshape(-1))
        assert np.array_equal(mc["nwhole"], z[q + "nwhole"].reshape(-1))
        assert np.array_equal(mc["nmovem"], z[q + "nmovem"].reshape(-1))
        assert_bits_equal(np.array([fadds, tr["faddbs"]], f32), np.array([z[q + "fadds"], z[q + "faddbs"]], f32),
                          f"cycle {c} fadds, faddbs")
        assert (ran1.idum, ran1.iy, ran1.mcall) == (int(z[q + "ran1_after_idum"]), int(z[q + "ran1_after_iy"]),
                                                     int(z[q + "ran1_after_mcall"]))


def load_shake(name="shake_rot.npz"):
    """tests/golden/shake_rot.npz (dih_shake.npz): the same box through two intramolecular cycles."""
    z = np.load(GOLDEN + "/" + name)
    box = BoxArrays.from_golden(z)
    for k in ("xa", "ya", "za", "xadd", "yadd", "zadd"):
        getattr(box, k)[:] = z["in_" + k]
    sc = z["scal"]
    model = dict(nbond=z["nbond"], iabond=z["iabond"], tbond=z["tbond"], amassa=z["amassa"], amassr=z["amassr"],
                 xav=z["xav"], xav1=z["xav1"], stepcl=sc[0], sizefactor=sc[1], tempb=sc[2], tempang=sc[3], simt=sc[4],
                 refine_intra=False, refine_intra_fac=f32(0.0), ngrot=z["ngrot"], dih=_dih(z))
    M = int(z["in_nnbrefmax"])
    n = int(z["in_nergpair"])
    st = dict(nnbrefmax=M, nergpair=n, nergpairm=np.ascontiguousarray(z["in_nergpairm"], np.int32),
              molergpair=np.ascontiguousarray(z["in_molergpair"][:M].T - 1, np.int32).reshape(-1),
              ergpairref=np.ascontiguousarray(z["in_ergpairref"][:M].T, np.int32).reshape(-1),
              ergpair=np.array(z["in_ergpair"][:n], f32))
    mc = dict(rejrate=f32(0.75), ireset=0, wholerot=np.array(z["wholerot_in"], f32),
              wholetrans=np.array(z["wholetrans_in"], f32), internrot=np.array(z["internrot_in"], f32),
              interntrans=np.array(z["interntrans_in"], f32), ngrot=np.array(z["ngrot"], np.int32))
    rot = dict(model=model, nrf=z["rot_nrf"], nrl=z["rot_nrl"], axis=z["rot_axis"].reshape(-1), first=z["rot_first"],
               last=z["rot_last"], atoms=z["rot_atoms"], stepri=f32(1.0))
    return z, box, st, mc, rot


@pytest.mark.parametrize("name", ["shake_rot.npz", "dih_shake.npz"])
def test_shake_rotation_golden_exercises_both_outcomes(name):
    z = np.load(GOLDEN + "/" + name)
    for c in range(int(z["cycles"])):
        ni, nm = z[f"c{c}_ninter"], z[f"c{c}_nmovei"]
        assert ni[0, 0] > 0 and 0 < ni[1, 0] < ni[0, 0]       # DMSO rotations tried, some rejected
        assert nm[0].sum() > 0 and nm[1].sum() > 0            # atom moves tried, some rejected


@pytest.mark.parametrize("name", ["shake_rot.npz", "dih_shake.npz"])
def test_shake_rotation_cycles_oracle_matches_reference(name):
    """The intramolecular cycle of a box with ROT (DIH) groups (molfit.py:124-267: atom moves, then
    the groups' rotations tested with the intermolecular change, molecules in index order), C
    restatement against the reference bit for bit over two cycles."""
    z, box, st, mc, rot = load_shake(name)
    ran1 = Ran1State.from_golden(z, "ran1_before_")
    fadds, faddbs, eo1 = f32(z["fadds_in"]), f32(z["faddbs_in"]), f32(0.0)
    for c in range(int(z["cycles"])):
        q = f"c{c}_"
        fadds, faddbs, nmovei, ninter, eo1, ran1, cosv = oracle.molfit_shake_rot(
            box, st, mc, rot, f32(z["stepmi"]), ran1, fadds, faddbs, eo1)
        assert_bits_equal(cosv, z[q + "cos"], f"cycle {c} cos")
        for k in ("xa", "ya", "za", "xadd", "yadd", "zadd"):
            assert_bits_equal(getattr(box, k), z[q + k], f"cycle {c} {k}")
        assert_bits_equal(st["ergpair"], z[q + "ergpair"], f"cycle {c} ergpair")
        for k in ("interntrans", "internrot", "wholerot", "wholetrans"):
            assert_bits_equal(mc[k], z[q + k], f"cycle {c} {k}")
        assert np.array_equal(nmovei, z[q + "nmovei"].reshape(-1))
        assert np.array_equal(ninter, z[q + "ninter"].reshape(-1))
        assert np.array_equal(mc["nstepreject"], z[q + "nstepreject"])
        assert_bits_equal(np.array([fadds, faddbs], f32), np.array([z[q + "fadds"], z[q + "faddbs"]], f32),
                          f"cycle {c} fadds, faddbs")
        assert (ran1.idum, ran1.iy, ran1.mcall) == (int(z[q + "ran1_after_idum"]), int(z[q + "ran1_after_iy"]),
                                                     int(z[q + "ran1_after_mcall"]))
        assert np.array_equal(ran1.iv, z[q + "ran1_after_iv"])
