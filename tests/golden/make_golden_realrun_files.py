"""Digests of every file the reference's own epsr program leaves in its shipped run folder
(EPSR-test: 200 DMSO + 400 water) after one unchanged run, made by running the reference
translation (epsr26) itself.

    EPSR_REFERENCE=<reference checkout> PYTHONDONTWRITEBYTECODE=1 python tests/golden/make_golden_realrun_files.py

The run folder is copied to a scratch directory and runepsr17 (epsr_standalone_rev3.py:1235)
runs on it as shipped: one iteration of five molfit calls (the intramolecular cycle first),
the refinement (atogen, gensq, the running sums, press, ptgnsq with its fits, generate_ep)
and the final output section (stog, the .erg/.g01/.f01/.pcof/.ato writers and the others).
tests/golden/realrun_files.json receives, for every file then in the folder, the SHA-256 of
its contents after ``normalised``: the run's date line of the .out file and the two elapsed-
time columns molfit's timers add to each line of fort.35 are the only parts that vary from run
to run, and are cut.  The output section's first stog call is captured on the way
(tests/golden/realrun_stog.npz, prefix st_).  About four minutes of CPU.
"""

from __future__ import annotations

import hashlib
import json
import os
import re
import shutil
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)
sys.path.insert(0, HERE)

import refstate  # noqa: E402

INPUT = "200DMSO400Water.EPSR.inp"
_DATE = re.compile(rb"^\s*Current date:.*$", re.M)
# fort.35 per molfit call: call, fadds, faddbs, then timer.sumtime1 and timer.sumtime2
_TIMERS = re.compile(rb"^(\s*\d+\s+\S+\s+\S+)\s+\d+\s+\d+\s*$", re.M)


def normalised(name, data):
    """The bytes of file ``name`` with the parts that vary between identical runs cut."""
    if name.endswith(".out"):
        return _DATE.sub(b"", data)
    if name == "fort.35":
        return _TIMERS.sub(rb"\1", data)
    return data


def output_digests(run):
    """SHA-256 of every file of the run folder, normalised, by name."""
    out = {}
    for name in sorted(os.listdir(run)):
        p = os.path.join(run, name)
        if os.path.isfile(p):
            with open(p, "rb") as f:
                out[name] = hashlib.sha256(normalised(name, f.read())).hexdigest()
    return out


def capture_stog(out, orig):
    """The output section's first stog call (ato_manipulation_rev4.py:4067, from
    epsr_standalone_rev3.py:2195: the fits to the data sets): rho, q, S(Q) (sets x Q points),
    r, the Q windows and xwt before; g(r) (sets x r points) after."""
    def wrapped(rho, q, sofq, r, gofr, nqmin, nqmax, nr, npairs, nqdim, nrdim, npdim, xwt):
        if "st_gofr" in out:
            return orig(rho, q, sofq, r, gofr, nqmin, nqmax, nr, npairs, nqdim, nrdim, npdim, xwt)
        ldq, n, nr = int(nqdim) + 1, int(npairs), int(nr)
        out["st_rho"] = np.float32(rho)
        out["st_q"] = np.array(q[:ldq], np.float32)
        out["st_sofq"] = np.ascontiguousarray(np.asarray(sofq)[:ldq, 1:n + 1].T, np.float32)
        out["st_r"] = np.array(r[: nr + 1], np.float32)
        out["st_nqmin"] = np.array(nqmin[1:n + 1], np.int32)
        out["st_nqmax"] = np.array(nqmax[1:n + 1], np.int32)
        out["st_xwt"] = np.array(xwt[1:n + 1], np.float32)
        res = orig(rho, q, sofq, r, gofr, nqmin, nqmax, nr, npairs, nqdim, nrdim, npdim, xwt)
        out["st_gofr"] = np.ascontiguousarray(np.asarray(gofr)[1:nr + 1, 1:n + 1].T, np.float32)
        return res
    return wrapped


def main():
    root = refstate.reference_root()
    work = tempfile.mkdtemp(prefix="epsr_realrun_files_")
    run = os.path.join(work, "EPSR-test")
    shutil.copytree(os.path.join(root, "EPSR-test"), run)
    refstate.load_reference(os.path.join(root, "src"))
    import importlib
    from epsr26.programs import run_program
    am = importlib.import_module("epsr26.library.ato_manipulation_rev4")
    st = {}
    orig = am.stog
    am.stog = capture_stog(st, orig)
    cwd = os.getcwd()
    os.chdir(run)
    try:
        rc = run_program("epsr", ["./", "epsr", INPUT])
    finally:
        os.chdir(cwd)
        am.stog = orig
    if rc not in (0, None):
        raise SystemExit(f"epsr ended with status {rc}")
    dig = output_digests(run)
    shutil.rmtree(work, ignore_errors=True)
    path = os.path.join(HERE, "realrun_files.json")
    with open(path, "w") as f:
        json.dump(dig, f, indent=1, sort_keys=True)
        f.write("\n")
    print("wrote", path, len(dig), "files")
    spath = os.path.join(HERE, "realrun_stog.npz")
    np.savez_compressed(spath, **st)
    print("wrote", spath, os.path.getsize(spath), "bytes")


if __name__ == "__main__":
    main()
