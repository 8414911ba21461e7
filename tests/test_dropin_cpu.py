"""Host logic of the drop-in layer (no GPU): the mapping from the reference's COMMON blocks
to the host box, installation onto the routine-owning modules, and the host fallbacks
for cycles outside the pair path (the reference's own routine runs, nothing on the device)."""

import numpy as np
import pytest

from epsr_python_translation_b200 import dropin
from epsr_python_translation_b200.box import BoxArrays
from tests import fake_common, goldens

f32 = np.float32


@pytest.mark.parametrize("case", goldens.CASES)
def test_box_from_common_matches_golden_box(case):
    z = goldens.load(case)
    p = dropin.PairPath(fake_common.common_from_golden(z), {})
    got, want = p.box_from_common(), BoxArrays.from_golden(z)
    for k, v in want.__dict__.items():
        g = getattr(got, k)
        if isinstance(v, np.ndarray):
            assert g.shape == v.shape and np.array_equal(g.view(np.uint8), np.ascontiguousarray(v, g.dtype).view(
                np.uint8)), k
        else:
            assert g == v, k
    assert got.stepcl == want.stepcl and got.sepmax == want.sepmax


def test_install_reroutes_and_uninstall_restores():
    z = goldens.load("c1_water")
    calls = []
    mods = fake_common.routine_modules(z, calls)
    before = {n: getattr(mods[dropin.OWNER[n]], n) for n in dropin.ROUTINES}
    p = dropin.PairPath(fake_common.common_from_golden(z), mods).install(dropin.ROUTINES)
    for n in dropin.ROUTINES:
        f = getattr(mods[dropin.OWNER[n]], n)
        assert f.__self__ is p and f.__name__ == n
    p.uninstall()
    for n in dropin.ROUTINES:
        assert getattr(mods[dropin.OWNER[n]], n) is before[n]
    p.install()
    assert set(p.orig) == set(dropin.DEFAULT_ROUTINES)


def test_cycles_without_bond_lists_or_group_tables_run_the_host_routine():
    """An intramolecular cycle when the COMMON blocks carry no bond lists, and internal
    rotations when they carry no group tables, keep the reference's own molfit."""
    z = goldens.load("mix_small")
    calls = []
    mods = fake_common.routine_modules(z, calls)
    c = fake_common.common_from_golden(z)
    dropin.PairPath(c, mods).install()
    # nisum >= intra: the shake / intramolecular branch (molfit.py:124-267)
    assert mods["molfit"].molfit(f32(0), f32(0), 100, 100, 5, 0) == (f32(0), f32(0), 1)
    # internal rotations due this cycle (molfit.py:290)
    c.molecom.stepri = f32(0.1)
    c.clustercom.ngrot[3] = 2
    mods["molfit"].molfit(f32(0), f32(0), 10, 100, 5, 0)
    assert calls == ["host:molfit", "host:molfit"]


@pytest.mark.parametrize("feature", ["coarsegraining", "threebody", "coord", "container", "tethered", "big"])
def test_features_outside_the_path_run_the_host_routines(feature):
    z = goldens.load("c1_water")
    calls = []
    mods = fake_common.routine_modules(z, calls)
    c = fake_common.common_from_golden(z)
    if feature == "coarsegraining":
        c.molecom_mod.coarsegraining = True
    elif feature == "threebody":
        c.threebody_mod.nthreeb = 1
    elif feature == "coord":
        c.coordconstraints_mod.ncoordconstraints = 2
    elif feature == "container":
        c.containerforces_mod.numcontainerforces = 1
    elif feature == "tethered":
        c.clustercom.tethered[5] = True
    else:
        c.clustercom.nato[2] = 65
    dropin.PairPath(c, mods).install()
    am = mods["ato_manipulation_rev4"]
    am.fmolec1(0, 0, f32(0), f32(0), f32(0), f32(0))
    mods["molfit"].molfit(f32(0), f32(0), 1, 100, 5, 0)
    am.atogen(None, 1000)
    assert calls == ["host:fmolec1", "host:molfit", "host:atogen"]
    if feature == "coarsegraining":
        mods["program"].gensq(10, None, None, None)
        assert calls[-1] == "host:gensq"


def test_cell_list_from_other_arrays_runs_the_host_routine():
    z = goldens.load("c1_water")
    calls = []
    mods = fake_common.routine_modules(z, calls)
    c = fake_common.common_from_golden(z)
    dropin.PairPath(c, mods).install()
    cc = c.clustercom
    mods["cellneighbourlist"].initialise_cellneighbourlist(10, cc.xadd.copy(), cc.yadd, cc.zadd, cc.nmol, f32(1))
    assert calls == ["host:initialise_cellneighbourlist"]


def test_fortran_helpers():
    assert [dropin._idiv(a, b) for a, b in ((7, 2), (-7, 2), (7, -2), (-7, -2), (0, 5))] == [3, -3, -3, 3, 0]
    a = dropin._fortran((3, 4), np.int32)
    assert a.shape == (4, 5) and a.flags.f_contiguous and not a.any()
    # the 32-bit device counter wraps; the reference's Python int does not
    assert dropin._mcall_advance(5, 12) == 12
    assert dropin._mcall_advance(2**32 + 5, 12) == 2**32 + 12
    assert dropin._mcall_advance(2**31 - 2, np.int32(-2**31 + 3)) == 2**31 + 3
    assert dropin._mcall_advance(3 * 2**32 - 1, 4) == 3 * 2**32 + 4


@pytest.mark.parametrize("name", ["rot.npz", "dih_rot.npz"])
def test_rotational_groups_and_dihedrals_from_common(name):
    """The rotational groups and their dihedral angles as the drop-in hands them to the device,
    read from COMMON blocks holding them as the reference does: the groups 0-based, each DIH
    group's dihedral atom pairs, and the glibc cosf/sinf of each angle -- the values the
    reference's en_dihedral computes (the golden's dih_cos/dih_sin), bit for bit."""
    z, c, mods, _ = fake_common.common_with_groups(name)
    p = dropin.PairPath(c, mods)
    nrf, nrl, axis, first, last, atoms = p._rot_groups()
    for got, want in ((nrf, z["rot_nrf"]), (nrl, z["rot_nrl"]), (axis, z["rot_axis"]), (first, z["rot_first"]),
                      (last, z["rot_last"]), (atoms, z["rot_atoms"])):
        assert np.array_equal(got, want)
    d = p._dihedrals()
    if name == "rot.npz":
        assert d is None
        return
    assert np.array_equal(d["grp_dih0"], z["dih_grp0"]) and np.array_equal(d["grp_isdih"], z["dih_isdih"])
    assert np.array_equal(d["dih_atoms"], z["dih_atoms"])
    assert np.array_equal(d["dih_cos"].view(np.uint32), z["dih_cos"].view(np.uint32))
    assert np.array_equal(d["dih_sin"].view(np.uint32), z["dih_sin"].view(np.uint32))
    assert d["tempdih"] == z["tempdih"]


def test_groups_of_another_type_run_the_host_routine():
    """A rotational group whose type is neither ROT nor DIH keeps the reference's own molfit."""
    z, c, mods, calls = fake_common.common_with_groups("rot.npz")
    c.molecom_mod.rotgrp[3] = "XYZ"
    p = dropin.PairPath(c, mods)
    assert p._rot_groups() is None
    p.install()
    mods["molfit"].molfit(f32(0), f32(0), 1, 100, 1, 0)
    assert calls == ["host:molfit"]
