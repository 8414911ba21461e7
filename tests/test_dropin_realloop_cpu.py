"""The drop-in inside the reference's own epsr loop: runepsr17 (epsr_standalone_rev3.py:1235)
runs unchanged on a copy of the reference's shipped run folder (EPSR-test: 200 DMSO + 400
water, the DMSO methyl groups as ROT groups) with dropin.install_reference(strict=True) in
place for every routine it installs by default -- the cell list, fmolec1, molfit, atogen,
press, gensq, sumgr, sumsq, stog, fit_expansion, generate_ep, generate_rp, each of which the
loop calls through its module (e.g. epsr_standalone_rev3.py:1265, :1280, :1318, :1343); the
reference's own routines are replaced by stubs that fail if the drop-in hands a call back to
them.  The device layer under the drop-in is the oracle-backed stand-in of
tests/oracle_device.py, so what runs here is the drop-in's own host side with the real epsr26
package: its COMMON modules and reset(), the loop's call order, the centres put back in the box
and fmolec1 called again after the intramolecular cycle, the refinement's ran1 draws.

The input file's niter is raised to 2 as for the fixture, so that the loop refines the
potential once through the drop-in (atogen, gensq, the running sums, press, ptgnsq's fits,
generate_ep) between the captures and the drop-in then sees the new tables.  Around the loop's first, second and sixth
molfit calls (the intramolecular cycle with the methyl rotations, a whole-molecule cycle, a
whole-molecule cycle with the methyl rotations) the COMMON state is captured as
tests/golden/make_golden_realrun.py captured it from the unmodified loop, and every array must
equal tests/golden/realrun.npz bit for bit: the box, the cell list and pair store the drop-in wrote, the step arrays, counters,
ran1 state, fadds/faddbs, and the coordinates and energies after each call.  The
loop's first cell list and the refinement's atogen, press, gensq, sumsq, sumgr, fit_expansion and generate_ep calls, as installed,
are captured the same way and must equal the reference's calls.  Only the scratch slot
ergold(1) is left out (the drop-in does not fill the reference's en_change work arrays).

A second run takes the shipped input file unchanged to its end (one iteration, then the final
output section with its four stog calls) and compares every file left in the run folder with
the unmodified run's (tests/golden/realrun_files.json, digests of the normalised bytes); its
first stog call, as installed, must equal the reference's (tests/golden/realrun_stog.npz).

Needs the reference checkout (EPSR_REFERENCE, the directory holding src/epsr26 and
EPSR-test); skipped without it.  About twenty seconds of CPU."""

import importlib
import json
import os
import shutil
import sys

import numpy as np
import pytest

from epsr_python_translation_b200 import dropin
from tests.goldens import GOLDEN, assert_bits_equal

ROOT = os.environ.get("EPSR_REFERENCE", "")
HAVE_REF = bool(ROOT) and os.path.isdir(os.path.join(ROOT, "src", "epsr26")) and \
    os.path.isdir(os.path.join(ROOT, "EPSR-test"))
ROUTINES = ("initialise_cellneighbourlist", "fmolec1", "molfit", "atogen", "press", "gensq", "sumgr", "sumsq",
            "stog", "fit_expansion", "generate_ep", "generate_rp")
SKIP = ("ergold1", "after_ergold1", "cos")


class _Stop(Exception):
    pass


def _host_routine(name):
    def f(*a, **k):
        raise AssertionError(f"the reference's own {name} ran: the drop-in routed it to the host")
    return f


def _install(tmp_path, monkeypatch):
    """The reference loaded, the stand-ins and the drop-in in place, the reference's own
    routines stubbed out, the run folder copied: (path, originals, journal, run folder)."""
    sys.path.insert(0, GOLDEN)
    import refstate
    from tests import oracle_device

    refstate.load_reference(os.path.join(ROOT, "src"))
    from epsr26.programs import load
    journal = oracle_device.install(monkeypatch)
    run = tmp_path / "EPSR-test"
    shutil.copytree(os.path.join(ROOT, "EPSR-test"), run)
    path = dropin.install_reference(load("epsr"), strict=True, routines=ROUTINES)
    real = dict(path.orig)
    for name in ROUTINES:
        path.orig[name] = _host_routine(name)
    return path, real, journal, run


def _run_program(run):
    from epsr26.programs import run_program
    cwd = os.getcwd()
    os.chdir(run)
    try:
        return run_program("epsr", ["./", "epsr", "200DMSO400Water.EPSR.inp"])
    finally:
        os.chdir(cwd)


def _run_loop_with_dropin(tmp_path, monkeypatch):
    sys.path.insert(0, GOLDEN)
    import make_golden_realrun as g

    path, real, journal, run = _install(tmp_path, monkeypatch)
    g.prepare_run(str(run))
    common = importlib.import_module("epsr26.common")
    mods = {"cellneighbourlist": importlib.import_module("epsr26.library.cellneighbourlist"),
            "ato_manipulation_rev4": importlib.import_module("epsr26.library.ato_manipulation_rev4"),
            "molfit": importlib.import_module("epsr26.library.molfit")}
    installed = mods["molfit"].molfit
    out, n = {}, {"n": 0, "taken": 0}

    def wrapped(fadds, faddbs, nisum, intra_, rotfreq, ireset):
        n["n"] += 1
        if n["n"] not in g.CAPTURE:
            return installed(fadds, faddbs, nisum, intra_, rotfreq, ireset)
        q = "k%d_" % n["taken"]
        g.snapshot(common, mods, out, q)
        g.intra_snapshot(common, out, q)
        out[q + "args"] = np.array([fadds, faddbs], np.float32)
        out[q + "args_int"] = np.array([nisum, intra_, rotfreq, ireset, n["n"]], np.int32)
        r = installed(fadds, faddbs, nisum, intra_, rotfreq, ireset)
        g.after(common, out, q, r, [])
        n["taken"] += 1
        if n["taken"] == len(g.CAPTURE):
            raise _Stop()
        return r

    mods["molfit"].molfit = wrapped
    # the refinement's routines, as installed, captured as the fixture captured the reference's
    am, program, cn = mods["ato_manipulation_rev4"], path.mods["program"], mods["cellneighbourlist"]
    inst = dict(cells=cn.initialise_cellneighbourlist, atogen=am.atogen, press=am.press, fit_expansion=program.fit_expansion,
                generate_ep=program.generate_ep, sumgr=program.sumgr, sumsq=program.sumsq, gensq=program.gensq)
    cn.initialise_cellneighbourlist = g.capture_cells(common, mods, out, inst["cells"])
    am.atogen = g.capture_atogen(common, mods, out, inst["atogen"])
    am.press = g.capture_press(common, mods, out, inst["press"])
    program.fit_expansion = g.capture_fit(common, out, inst["fit_expansion"])
    program.generate_ep = g.capture_generate_ep(common, out, inst["generate_ep"])
    program.sumgr, program.sumsq = g.capture_sums(common, out, inst["sumgr"], inst["sumsq"])
    program.gensq = g.capture_gensq(common, out, inst["gensq"])
    try:
        _run_program(run)
    except _Stop:
        pass
    finally:
        mods["molfit"].molfit = installed
        am.atogen, am.press = inst["atogen"], inst["press"]
        cn.initialise_cellneighbourlist = inst["cells"]
        for k in ("fit_expansion", "generate_ep", "sumgr", "sumsq", "gensq"):
            setattr(program, k, inst[k])
        path.orig = real
        path.uninstall()
    return out, journal


def _run_program_with_dropin(tmp_path, monkeypatch):
    """The shipped run to its end through the drop-in: the digests of the files it leaves."""
    sys.path.insert(0, GOLDEN)
    import make_golden_realrun_files as gf

    path, real, journal, run = _install(tmp_path, monkeypatch)
    am = importlib.import_module("epsr26.library.ato_manipulation_rev4")
    stog, st = am.stog, {}
    am.stog = gf.capture_stog(st, stog)
    try:
        rc = _run_program(run)
    finally:
        am.stog = stog
        path.orig = real
        path.uninstall()
    assert rc in (0, None)
    return gf.output_digests(str(run)), journal, st


@pytest.mark.skipif(not HAVE_REF, reason="needs the reference checkout (EPSR_REFERENCE)")
def test_dropin_in_the_reference_loop_matches_the_unmodified_loop(tmp_path, monkeypatch):
    z = np.load(os.path.join(GOLDEN, "realrun.npz"))
    out, calls = _run_loop_with_dropin(tmp_path, monkeypatch)
    assert set(ROUTINES) == set(dropin.DEFAULT_ROUTINES)
    # routed as the loop asks: the EP at set-up; the cell list and store, the intramolecular
    # cycle, the store again, four whole-molecule cycles; the refinement (atogen, gensq, the
    # running sums, press, one fit per data set, generate_ep); then, the lattice rebuilt (its
    # float cos(90 deg) entries become exact zeros, so the drop-in makes a new device box), the
    # cell list, the store and a fifth whole-molecule cycle, with rotations.  stog (the output
    # section) and generate_rp (the multiply_pcoefex command) are not reached before it.
    assert calls == ["generate_ep", "box", "cell_list", "en_mole_intra", "fmolec1", "molfit_shake", "en_mole_intra",
                     "fmolec1"] + ["molfit"] * 4 + ["atogen", "gensq", "sumsq", "sumgr", "press"] + \
        ["fit_expansion"] * 3 + ["generate_ep", "box", "cell_list", "en_mole_intra", "fmolec1", "molfit"], calls
    checked = 0
    for key, v in out.items():
        if any(key.endswith("_" + s) for s in SKIP):
            continue
        assert key in z.files, key
        ref = z[key]
        a = np.asarray(v)
        if a.dtype.kind == "f":
            assert_bits_equal(a, ref, key)
        else:
            assert a.shape == ref.shape and np.array_equal(a, ref), key
        checked += 1
    assert checked > 100
    for q in ("k0_", "k1_", "k2_"):
        assert int(out[q + "ran1_after_mcall"]) > int(out[q + "ran1_before_mcall"])


@pytest.mark.skipif(not HAVE_REF, reason="needs the reference checkout (EPSR_REFERENCE)")
def test_dropin_in_the_reference_loop_writes_the_unmodified_runs_files(tmp_path, monkeypatch):
    """The shipped run (one iteration, then the final output section) to its end through the
    drop-in: every file it leaves in the run folder -- .erg, .g01, .f01, .pcof, the .ato and
    the rest, 66 files -- has the bytes the unmodified run left (tests/golden/realrun_files.json
    from tests/golden/make_golden_realrun_files.py), the run date and molfit's elapsed-time
    columns excepted."""
    with open(os.path.join(GOLDEN, "realrun_files.json")) as f:
        want = json.load(f)
    got, calls, st = _run_program_with_dropin(tmp_path, monkeypatch)
    assert sorted(got) == sorted(want)
    bad = [k for k in want if got[k] != want[k]]
    assert not bad, bad
    for k in ("200DMSO400Water.EPSR.erg", "200DMSO400Water.EPSR.g01", "200DMSO400Water.EPSR.f01",
              "200DMSO400Water.pcof", "200DMSO400Water.ato"):
        assert k in want
    # the output section's four transforms ran through the drop-in too; the first as the reference's
    z = np.load(os.path.join(GOLDEN, "realrun_stog.npz"))
    assert sorted(st) == sorted(z.files)
    for k in z.files:
        if z[k].dtype.kind == "f":
            assert_bits_equal(st[k], z[k], k)
        else:
            assert np.array_equal(st[k], z[k]), k
    assert calls.count("stog") == 4 and calls.count("molfit") == 4 and calls.count("molfit_shake") == 1, calls


def test_oracle_stand_ins_keep_the_device_layers_signatures():
    """Every stand-in of tests/oracle_device.py takes the arguments of the device-layer call it
    replaces (device.DeviceBox, intra.IntraModel, transforms, potential.generate_ep), so the
    drop-in calls both alike.  Needs no reference checkout."""
    import inspect

    from epsr_python_translation_b200 import device, intra, potential, transforms
    from tests import oracle_device as od

    def params(f):
        return [(p.name, p.kind, p.default) for p in inspect.signature(f).parameters.values()]

    pairs = [(getattr(od.OracleDeviceBox, n), getattr(device.DeviceBox, n))
             for n in ("upload", "upload_coords", "download_coords", "ran1_tensor", "cell_list", "download_cells",
                       "fmolec1", "download_store", "mc_setup", "set_rotations", "set_cos_override", "molfit",
                       "check_status", "download_mc", "atogen", "download_wav", "press")]
    pairs += [(getattr(od.OracleIntraModel, n), getattr(intra.IntraModel, n))
              for n in ("__init__", "en_mole_intra", "molfit_shake")]
    pairs += [(getattr(od, n), getattr(transforms, n)) for n in ("gensq", "sumgr", "sumsq", "stog", "fit_expansion")]
    pairs += [(od.generate_ep, potential.generate_ep)]
    bad = [f"{a.__qualname__}: {params(a)} vs {params(b)}" for a, b in pairs if params(a) != params(b)]
    assert not bad, "\n".join(bad)
