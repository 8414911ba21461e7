"""The potential refinement of ptgnsq (epsr_standalone_rev3.py:3790-4021) on the device, stage by
stage through the C ABI -- epsr_ptgnsq_difference (real*8 weights), epsr_fit_expansion_batch
(both data sets on one ran1 stream), epsr_ep_update, the host basis builder and
epsr_generate_ep(changepotfac off) -- against the reference's own ptgnsq run on seeded state
(tests/golden/ptgnsq.npz), bit for bit, ran1 stream included."""

import numpy as np
import pytest
import torch

from tests.goldens import assert_bits_equal
from tests.test_ptgnsq_oracle import CASES, TABS, check_refined, load

pytestmark = pytest.mark.gpu
f32 = np.float32


def _dev(a, dtype=torch.float32):
    return torch.from_numpy(np.ascontiguousarray(a)).to(device="cuda", dtype=dtype)


@pytest.mark.parametrize("name", CASES)
def test_ptgnsq_refinement_device_matches_reference(name):
    from epsr_python_translation_b200 import potential, transforms
    from epsr_python_translation_b200.box import Ran1State
    z, n = load(name)
    dt = transforms.ptgnsq_difference(_dev(z["data"]), _dev(z["cwt"], torch.float64), _dev(z["qwind"]), q=z["q"],
                                      nqmin=n["nqmin"], nqmax=n["nqmax"], szeros=n["szeros"], qmin=n["qmin"],
                                      wq=_dev(z["wq"], torch.float64), xray=z["xray"])
    expr = np.concatenate([np.zeros(1, f32), z["expsq"]])
    ran1 = _dev(Ran1State.from_golden(z, "ran1_before_").as_array(), torch.int32)
    res = transforms.fit_expansion_batch(dt, expr, z["pcoefd_in"], z["pstepd_in"], 1, n["nq"], 1, n["nterms"],
                                         n["nits"], 10, ran1, strict=True)
    fits = res["wtold"]
    pcoefd = z["pcoefd_in"].copy()
    pcoefd[:, 2:] = fits.cpu().numpy()[:, 2:]
    dmax, absolute_energy, erequnit, ereqstep, potfacamp, potfac, _ = (f32(v) for v in z["scal"])
    pc = _dev(z["pcoefp_in"])
    potential.ep_update(pc, z["iref"], _dev(z["efacp"]), _dev(z["cwtpot"], torch.float64), fits, potfac)
    pdmin, pdstep, pdmax, psigma2, rho = (f32(v) for v in z["basis"])
    expgr, _ = potential.basis(n["npt2"], n["nterms"], z["x"], False, pdmin, pdstep, pdmax, psigma2, rho, 0.0)
    tabs = {k: _dev(z["in_" + k]) for k in TABS}
    pw = torch.zeros(n["nterms"] + 1, device="cuda")
    potential.generate_ep(n["npt"], n["npt2"], n["nterms"], _dev(expgr), pc, z["iref"], dmax, _dev(z["xstar"]),
                          _dev(z["wfac"]), _dev(z["in_ecoul"]), tabs, pw, absolute_energy, erequnit, ereqstep,
                          potfacamp, _dev([potfac]), changepotfac=False)
    torch.cuda.synchronize()
    got = dict(pcoefd=pcoefd, pstepd=res["stepr"], potnoi=res["chisq"], pcoefp=pc.cpu().numpy(),
               pwtold=pw.cpu().numpy(), tabs={k: v.cpu().numpy() for k, v in tabs.items()})
    check_refined(got, z, n, "device")
    r = ran1.cpu().numpy()
    assert int(r[0]) == int(z["ran1_after_idum"]) and int(r[1]) == int(z["ran1_after_iy"])
    assert np.array_equal(r[3:], z["ran1_after_iv"])
    assert_bits_equal(np.array(int(r[2]), np.int32), np.array(np.int64(z["ran1_after_mcall"]).astype(np.int32)),
                      "mcall")
