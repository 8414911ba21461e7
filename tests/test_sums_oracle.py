"""The C restatement of the running averages sumgr and sumsq (epsr_standalone_rev3.py:3578-3677)
against the reference's own sumgr/sumsq run on seeded state (tests/golden/sums.npz, made by
tests/golden/make_golden_sums.py), bit for bit over consecutive calls."""

import numpy as np
import pytest

from oracle import oracle
from tests.goldens import GOLDEN, assert_bits_equal

GR = ("gorintra", "gorinter", "gr2intra", "gr2inter")
SQ = ("soqintra", "soqinter", "sq2intra", "sq2inter")


def case_arrays(z, name):
    """The golden case in the device layout: accumulators (npairs, ld), samples (2, npairs, ld)."""
    npairs, nz, nq, ncalls = (int(v) for v in z[f"{name}_dims"])
    acc = {k: np.ascontiguousarray(z[f"{name}_in_{k}"].T) for k in GR + SQ}
    acc["entsig"] = np.zeros((npairs, nz + 1), np.float32)
    fc1, fc2 = (float(v) for v in z[f"{name}_fc"])
    calls = []
    for c in range(ncalls):
        wav = np.ascontiguousarray(z[f"{name}_c{c}_wav"].transpose(0, 2, 1))
        qw = np.ascontiguousarray(z[f"{name}_c{c}_qwind"].transpose(0, 2, 1))
        want = {k: np.ascontiguousarray(z[f"{name}_c{c}_{k}"].T) for k in GR + SQ + ("entsig",)}
        calls.append((wav, qw, want))
    return dict(npairs=npairs, nz=nz, nq=nq, acc=acc, fc=(fc1, fc2), calls=calls, ycoh=z[f"{name}_ycoh"])


@pytest.mark.parametrize("name", ["small", "mix"])
def test_running_sums_oracle_matches_reference(name):
    z = np.load(GOLDEN + "/sums.npz")
    c = case_arrays(z, name)
    acc = c["acc"]
    for i, (wav, qw, want) in enumerate(c["calls"]):
        g = oracle.sumgr(c["nz"], wav, c["ycoh"], *c["fc"], acc)
        q = oracle.sumsq(c["nq"], qw, *c["fc"], acc)
        acc = {**acc, **g, **q}
        for k in GR + ("entsig",):
            assert_bits_equal(acc[k][:, 1: c["nz"] + 1], want[k][:, 1: c["nz"] + 1], f"{name} call {i} {k}")
        for k in SQ:
            assert_bits_equal(acc[k][:, 1: c["nq"] + 1], want[k][:, 1: c["nq"] + 1], f"{name} call {i} {k}")
