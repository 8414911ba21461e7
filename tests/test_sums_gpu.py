"""The running averages sumgr and sumsq (epsr_standalone_rev3.py:3578-3677) on the device,
through the C ABI and through the drop-in wrappers with the reference's signatures, against
the reference's own sumgr/sumsq run on seeded state (tests/golden/sums.npz), bit for bit over
consecutive calls."""

from types import SimpleNamespace as NS

import numpy as np
import pytest
import torch

from tests.goldens import GOLDEN, assert_bits_equal
from tests.test_sums_oracle import GR, SQ, case_arrays

pytestmark = pytest.mark.gpu
f32 = np.float32


@pytest.mark.parametrize("name", ["small", "mix"])
def test_running_sums_device_match_reference(name):
    from epsr_python_translation_b200 import transforms
    z = np.load(GOLDEN + "/sums.npz")
    c = case_arrays(z, name)
    dev = {k: torch.from_numpy(v.copy()).cuda() for k, v in c["acc"].items()}
    yc = torch.from_numpy(np.ascontiguousarray(c["ycoh"], f32)).cuda()
    fc1, fc2 = c["fc"]
    for i, (wav, qw, want) in enumerate(c["calls"]):
        transforms.sumgr(c["nz"], torch.from_numpy(wav.reshape(-1)).cuda(), yc, fc1, fc2, dev)
        transforms.sumsq(c["nq"], torch.from_numpy(qw.reshape(-1)).cuda(), fc1, fc2, dev)
        for k in GR + ("entsig",):
            assert_bits_equal(dev[k].cpu().numpy()[:, 1: c["nz"] + 1], want[k][:, 1: c["nz"] + 1],
                              f"{name} call {i} {k}")
        for k in SQ:
            assert_bits_equal(dev[k].cpu().numpy()[:, 1: c["nq"] + 1], want[k][:, 1: c["nq"] + 1],
                              f"{name} call {i} {k}")


def test_running_sums_dropin_match_reference():
    """PairPath.sumgr(nz, wav) / sumsq(nq, qwind) on COMMON-style 1-based arrays."""
    from epsr_python_translation_b200 import dropin
    z = np.load(GOLDEN + "/sums.npz")
    name = "mix"
    c = case_arrays(z, name)
    npairs, nz, nq = c["npairs"], c["nz"], c["nq"]
    mpz, mpts = nz + 8, nq + 8
    e16 = NS(ycoh=np.zeros(mpz, f32))
    e16.ycoh[: nz + 1] = c["ycoh"]
    for k in GR + ("entsig",):
        a = np.zeros((mpz, npairs + 1), f32, order="F")
        a[: nz + 1, 1:] = c["acc"][k].T
        setattr(e16, k, a)
    for k in SQ:
        a = np.zeros((mpts, npairs + 1), f32, order="F")
        a[: nq + 1, 1:] = c["acc"][k].T
        setattr(e16, k, a)
    common = NS(epsr16=e16, molecom=NS(npairs=npairs), sumvalues=NS(fc1=c["fc"][0], fc2=c["fc"][1]))
    path = dropin.PairPath(common, {})
    for i, (wav, qw, want) in enumerate(c["calls"]):
        w = np.zeros((3, mpz, npairs + 1), f32, order="F")
        w[1:3, : nz + 1, 1:] = wav.transpose(0, 2, 1)
        q = np.zeros((3, mpts, npairs + 1), f32, order="F")
        q[1:3, : nq + 1, 1:] = qw.transpose(0, 2, 1)
        assert path.sumgr(nz, w) is None
        assert path.sumsq(nq, q) is None
        for k in GR + ("entsig",):
            assert_bits_equal(getattr(e16, k)[1: nz + 1, 1:], want[k][:, 1: nz + 1].T, f"call {i} {k}")
        for k in SQ:
            assert_bits_equal(getattr(e16, k)[1: nq + 1, 1:], want[k][:, 1: nq + 1].T, f"call {i} {k}")
