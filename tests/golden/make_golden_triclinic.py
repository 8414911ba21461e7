"""Golden vectors for the triclinic minimum image (minimagec.py:13-45, minimage :48-62).

    EPSR_REFERENCE=<reference checkout> PYTHONDONTWRITEBYTECODE=1 python tests/golden/make_golden_triclinic.py

Runs the reference's own minimagec with lattice.cubic False on three seeded lattices (a
monoclinic cell, a general triclinic cell, and a cubic cell built from angles whose
off-diagonal components are cos(90 deg) rounding residues rather than zeros, as the reference's
lattice set-up leaves them) over 2,000 seeded points each, spread over several box lengths so
that every image shift occurs.  Writes tests/golden/triclinic.npz: per lattice the six
components {alatx, blatx, clatx, blaty, claty, clatz} (float32), the points and the
reference's results.
"""

from __future__ import annotations

import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import refstate  # noqa: E402

f32 = np.float32


def lattice_from_angles(a, b, c, alpha, beta, gamma):
    """Lattice vectors from lengths and angles in float32 (a along x, b in the xy plane), the
    usual construction, scaled so that blaty = 1 (box-fraction units)."""
    ca, cb, cg = (f32(math.cos(math.radians(t))) for t in (alpha, beta, gamma))
    sg = f32(math.sin(math.radians(gamma)))
    alatx = f32(a)
    blatx, blaty = f32(b) * cg, f32(b) * sg
    clatx = f32(c) * cb
    claty = f32(c) * (ca - cb * cg) / sg
    clatz = f32(math.sqrt(max(float(f32(c) * f32(c) - clatx * clatx - claty * claty), 0.0)))
    v = np.array([alatx, blatx, clatx, blaty, claty, clatz], f32)
    return (v / blaty).astype(f32)


def main():
    refstate.load_reference()
    from epsr26 import common
    from epsr26.common import lattice
    from epsr26.library import minimagec
    common.reset()
    cases = {
        "mono": lattice_from_angles(20.0, 22.0, 25.0, 90.0, 105.0, 90.0),
        "tric": lattice_from_angles(20.0, 23.0, 27.0, 80.0, 95.0, 110.0),
        "cubic_angles": lattice_from_angles(20.0, 20.0, 20.0, 90.0, 90.0, 90.0),
    }
    out = {}
    rng = np.random.default_rng(11)
    for name, v in cases.items():
        lattice.cubic = False
        lattice.alatx, lattice.blatx, lattice.clatx, lattice.blaty, lattice.claty, lattice.clatz = (f32(t) for t in v)
        pts = rng.uniform(-2.5, 2.5, size=(2000, 3)).astype(f32)
        res = np.zeros_like(pts)
        for k in range(pts.shape[0]):
            x, y, z = minimagec.minimagec(f32(pts[k, 0]), f32(pts[k, 1]), f32(pts[k, 2]))
            res[k] = (x, y, z)
        out[f"{name}_lat6"] = v
        out[f"{name}_pts"] = pts
        out[f"{name}_out"] = res
    out["cases"] = np.array(list(cases))
    np.savez_compressed(os.path.join(HERE, "triclinic.npz"), **out)
    print("wrote triclinic.npz", {k: cases[k].tolist() for k in cases})


if __name__ == "__main__":
    main()
