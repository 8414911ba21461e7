"""Golden vectors for the running averages sumgr and sumsq (epsr_standalone_rev3.py:3578-3637
and :3642-3677), made by running the reference translation (epsr26) on seeded state.

Run in a container where the reference is importable (it is read-only; nothing is written
there):

    EPSR_REFERENCE=<reference checkout> PYTHONDONTWRITEBYTECODE=1 python tests/golden/make_golden_sums.py

For each case the accumulators (gorintra/gorinter/gr2intra/gr2inter, soqintra/...) are
filled with seeded running values, the new histograms wav(2, nz, npairs) and S(Q)
qwind(2, nq, npairs) with seeded samples (some ycoh <= 0 to exercise that branch), fc1, fc2
set as runepsr17 sets them for a given nsum (:1614-1615), and sumgr/sumsq called a few times
in a row.  tests/golden/sums.npz receives, per case prefix, the inputs and the arrays after
each call (0-based arrays, r or Q index first as in the reference: [j, pair]).
"""

from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import refstate  # noqa: E402

f32 = np.float32
REF = refstate.reference_root()


def run_case(name, npairs, nz, nq, nsum, ncalls, seed, out):
    from epsr26.common import epsr16, molecom, sumvalues
    rng = np.random.default_rng(seed)
    molecom.npairs = npairs
    ycoh = (rng.uniform(0.0, 4.0, nz + 1)).astype(f32)
    ycoh[rng.integers(2, nz + 1, 5)] = f32(0.0)        # the ycoh <= 0 branch
    epsr16.ycoh[: nz + 1] = ycoh
    acc = {}
    for k in ("gorintra", "gorinter", "gr2intra", "gr2inter"):
        v = (rng.uniform(0.0, 2.0, (nz + 1, npairs))).astype(f32)
        getattr(epsr16, k)[1: nz + 1, 1: npairs + 1] = v[1:]
        acc[k] = v
    for k in ("soqintra", "soqinter", "sq2intra", "sq2inter"):
        v = (rng.standard_normal((nq + 1, npairs)) * 0.3).astype(f32)
        if k.startswith("sq2"):
            v = np.abs(v)
        getattr(epsr16, k)[1: nq + 1, 1: npairs + 1] = v[1:]
        acc[k] = v
    for k, v in acc.items():
        out[f"{name}_in_{k}"] = v
    out[f"{name}_ycoh"] = ycoh
    sumvalues.fc1 = float(f32(1.0) / f32(nsum))
    sumvalues.fc2 = float(f32(nsum - 1)) * sumvalues.fc1
    out[f"{name}_fc"] = np.array([sumvalues.fc1, sumvalues.fc2])
    from epsr26.fortran.arrays import real_array
    for c in range(ncalls):
        wav_in = (rng.uniform(0.0, 3.0, (2, nz + 1, npairs))).astype(f32)
        q_in = (rng.standard_normal((2, nq + 1, npairs)) * 0.5).astype(f32)
        wav = real_array(2, nz, npairs)
        wav[1:3, 1: nz + 1, 1: npairs + 1] = wav_in[:, 1:, :]
        qwind = real_array(2, nq, npairs)
        qwind[1:3, 1: nq + 1, 1: npairs + 1] = q_in[:, 1:, :]
        out[f"{name}_c{c}_wav"] = wav_in
        out[f"{name}_c{c}_qwind"] = q_in
        refstate_ep.sumgr(nz, wav)
        refstate_ep.sumsq(nq, qwind)
        for k in ("gorintra", "gorinter", "gr2intra", "gr2inter", "entsig"):
            out[f"{name}_c{c}_{k}"] = np.array(getattr(epsr16, k)[: nz + 1, : npairs + 1], f32)[:, 1:]
        for k in ("soqintra", "soqinter", "sq2intra", "sq2inter"):
            out[f"{name}_c{c}_{k}"] = np.array(getattr(epsr16, k)[: nq + 1, : npairs + 1], f32)[:, 1:]
    out[f"{name}_dims"] = np.array([npairs, nz, nq, ncalls])
    print(f"[{name}] done", flush=True)


refstate_ep = None

if __name__ == "__main__":
    common, ep = refstate.load_reference(os.path.join(REF, "src"))
    common.reset()
    import importlib
    refstate_ep = importlib.import_module("epsr26.programs.epsr_standalone_rev3")
    out = {}
    run_case("small", npairs=3, nz=240, nq=600, nsum=5, ncalls=3, seed=1, out=out)
    run_case("mix", npairs=21, nz=530, nq=600, nsum=10, ncalls=2, seed=2, out=out)
    path = os.path.join(HERE, "sums.npz")
    np.savez_compressed(path, **out)
    print("wrote", path)
