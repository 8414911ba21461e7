"""Golden vectors for press (ato_manipulation_rev4.py:3903-4062), made by running the
reference translation (epsr26) on the golden systems.

Run in a container where the reference is importable (it is read-only; nothing is written
there):

    EPSR_REFERENCE=<reference checkout> PYTHONDONTWRITEBYTECODE=1 python tests/golden/make_golden_press.py [case ...]

For each case the system is rebuilt with the seed that make_golden.py used, the cell list
and the pair store are made by the reference (initialise_cellneighbourlist, fmolec1) as in
make_golden.py, and press is called at those coordinates with one data file of unit weight
(energf/pressf set to known values, so their rescaling is checked too) and no EP coefficient
sets (abs_energy_ep returns 0).  tests/golden/press.npz receives, per case prefix:

* ``<case>_volume``, ``<case>_simt``: the inputs press reads besides the store;
* ``<case>_nergpair``: the store size, to check that the store matches <case>.npz;
* ``<case>_energy``, ``<case>_pressc``: press's results;
* ``<case>_energf_in``, ``<case>_pressf_in``, ``<case>_energf``, ``<case>_pressf``: the
  per-file values before and after press rescales them.
"""

from __future__ import annotations

import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)
sys.path.insert(0, HERE)

from epsr_python_translation_b200 import configs  # noqa: E402
import refstate  # noqa: E402

f32 = np.float32
REF = refstate.reference_root()


def run_press(name, s, out, *, rejrate=0.75, nmolcell=10):
    from epsr26.common import clustercom, epsr16, molecom, potential_par
    from epsr26.fortran import f32 as F, r4
    from epsr26.fortran.arrays import real_array
    from epsr26.library import ato_manipulation_rev4, cellneighbourlist, minimagec, molfit

    t0 = time.time()
    nmt = s.nmoltype
    refstate.populate(s, rejrate=rejrate, wholerot=[0.0556] * nmt, wholetrans=[f32(0.5) / s.dmax] * nmt)
    clustercom.volume = f32(s.L ** 3)
    # cell list and store exactly as make_golden.py:run_case
    sepmax = epsr16.xstar[epsr16.nptmax] + molecom.maxmolsize + r4(3.0) / clustercom.dmax
    cellneighbourlist.initialise_cellneighbourlist(nmolcell, clustercom.xadd, clustercom.yadd, clustercom.zadd,
                                                   clustercom.nmol, sepmax)
    for im in range(1, s.nmol + 1):
        clustercom.xadd[im], clustercom.yadd[im], clustercom.zadd[im] = minimagec.minimagec(
            clustercom.xadd[im], clustercom.yadd[im], clustercom.zadd[im])
    ato_manipulation_rev4.fmolec1(0, 0, F(0), F(0), F(0), F(0))
    del molfit  # (en_mole_intra is called inside fmolec1)
    from epsr26.common import ergpairreference as erd
    print(f"[{name}] fmolec1 done {time.time() - t0:.1f}s", flush=True)
    # one data file of unit weight, no EP coefficient sets
    epsr16.nfile = 1
    potential_par.wsum[1] = f32(1.0)
    potential_par.npairspcof = 0
    energf = real_array(4)
    pressf = real_array(4)
    energf[1] = f32(12.5)
    pressf[1] = f32(-3.25)
    ef_in, pf_in = f32(energf[1]), f32(pressf[1])
    energy, pressc, energabs, energthreeb, prthreebout = ato_manipulation_rev4.press(
        F(0), F(0), energf, pressf, F(0), F(0), F(0))
    out[name + "_volume"] = np.float32(clustercom.volume)
    out[name + "_simt"] = np.float32(molecom.simt)
    out[name + "_nergpair"] = np.int64(erd.nergpair)
    out[name + "_energy"] = np.float32(energy)
    out[name + "_pressc"] = np.float32(pressc)
    out[name + "_energabs"] = np.float32(energabs)
    out[name + "_energf_in"] = ef_in
    out[name + "_pressf_in"] = pf_in
    out[name + "_energf"] = np.float32(energf[1])
    out[name + "_pressf"] = np.float32(pressf[1])
    print(f"[{name}] press done {time.time() - t0:.1f}s energy={energy} pressc={pressc}", flush=True)


CASES = {
    "c1_water": lambda o: run_press("c1_water", configs.c1_water(seed=1), o),
    "mix_small": lambda o: run_press("mix_small", configs.c2_mixture(seed=3, ndmso=20, nwater=40), o),
    "silica": lambda o: run_press("silica", configs.silica(seed=4, natom=240), o),
    "c2_mixture": lambda o: run_press("c2_mixture", configs.c2_mixture(seed=1), o),
}


if __name__ == "__main__":
    refstate.load_reference(os.path.join(REF, "src"))
    path = os.path.join(HERE, "press.npz")
    out = dict(np.load(path)) if os.path.exists(path) else {}
    for n in sys.argv[1:] or list(CASES):
        CASES[n](out)
    np.savez_compressed(path, **out)
    print("wrote", path)
