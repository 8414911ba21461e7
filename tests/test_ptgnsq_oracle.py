"""The potential refinement of ptgnsq (epsr_standalone_rev3.py:3790-4021) restated by the oracle
-- the data-set differences with real*8 weights, one fit_expansion per data set, the
coefficient increment (:3948-3962) and generate_ep(.false.) (:4014) -- against the reference's
own ptgnsq run on seeded state (tests/golden/ptgnsq.npz, made by
tests/golden/make_golden_ptgnsq.py), bit for bit, ran1 stream included."""

import numpy as np
import pytest

from epsr_python_translation_b200.box import Ran1State
from oracle import oracle
from tests.goldens import GOLDEN, assert_bits_equal

f32 = np.float32
TABS = ("xavs", "xavs1", "xavtot", "xavtot1")


CASES = ["ptgnsq", "ptgnsq_window", "ptgnsq_xray"]


def load(name="ptgnsq"):
    z = np.load(GOLDEN + f"/{name}.npz")
    npairs, nsets, nfile, nq, nterms, nits, npt, npt2 = (int(v) for v in z["dims"])
    w = z["window"]
    return z, dict(npairs=npairs, nsets=nsets, nfile=nfile, nq=nq, nterms=nterms, nits=nits, npt=npt, npt2=npt2,
                   qmin=f32(w[0]), nqmin=w[1: 1 + nfile].astype(np.int32), szeros=w[1 + nfile: 1 + 2 * nfile],
                   nqmax=np.full(nfile, nq, np.int32))


def refine_oracle(z, n):
    """The oracle's chain on the golden inputs; returns the refined state."""
    dt = oracle.ptgnsq_difference(z["data"], z["cwt"], z["qwind"], z["q"], n["nqmin"], n["nqmax"], n["szeros"],
                                  n["qmin"], z["wq"], z["xray"])
    expr = np.concatenate([np.zeros(1, f32), z["expsq"]])
    ran1 = Ran1State.from_golden(z, "ran1_before_")
    pcoefd = z["pcoefd_in"].copy()
    pstepd = z["pstepd_in"].copy()
    potnoi = np.zeros(n["nfile"], f32)
    fits = np.zeros((n["nfile"], n["nterms"] + 1), f32)
    for d in range(n["nfile"]):
        res, ran1 = oracle.fit_expansion(dt[d], expr, pcoefd[d], pstepd[d], 1, n["nq"], 1, n["nterms"], n["nits"], 10,
                                         ran1)
        fits[d] = res["wtold"]
        pcoefd[d, 2:] = res["wtold"][2:]
        pstepd[d] = res["stepr"]
        potnoi[d] = res["chisq"]
    dmax, absolute_energy, erequnit, ereqstep, potfacamp, potfac, _ = (f32(v) for v in z["scal"])
    pc = oracle.ep_update(z["pcoefp_in"], z["iref"], z["efacp"], z["cwtpot"], fits, potfac)
    pdmin, pdstep, pdmax, psigma2, rho = (f32(v) for v in z["basis"])
    expgr = oracle.calc_pwrexpr_grad(n["npt2"], n["nterms"], pdmin, pdstep, pdmax, psigma2, rho, z["x"])
    tabs = {k: z["in_" + k] for k in TABS}
    tabs, pc, pw, _, _, _ = oracle.generate_ep(n["npt"], n["npt2"], n["nterms"], expgr, pc, z["iref"], dmax, z["xstar"],
                                               z["wfac"], z["in_ecoul"], tabs, np.zeros(n["nterms"] + 1, f32),
                                               np.array([absolute_energy, erequnit, ereqstep, potfacamp], f32),
                                               potfac, False)
    return dict(dt=dt, pcoefd=pcoefd, pstepd=pstepd, potnoi=potnoi, pcoefp=pc, pwtold=pw, tabs=tabs, ran1=ran1)


def check_refined(got, z, n, who):
    for k in ("pstepd", "potnoi"):
        assert_bits_equal(np.asarray(got[k], f32), z[k], f"{who} {k}")
    assert_bits_equal(got["pcoefd"][:, 2: n["nterms"] + 1], z["pcoefd"][:, 2: n["nterms"] + 1], f"{who} pcoefd")
    assert_bits_equal(got["pcoefp"][:, 1: n["nterms"] + 1], z["pcoefp"][:, 1:], f"{who} pcoefp")
    assert_bits_equal(got["pwtold"][1: n["nterms"] + 1], z["pwtold"][1:], f"{who} pwtold")
    for k in TABS:
        assert_bits_equal(got["tabs"][k], z[k], f"{who} {k}")


@pytest.mark.parametrize("name", CASES)
def test_ptgnsq_refinement_oracle_matches_reference(name):
    z, n = load(name)
    got = refine_oracle(z, n)
    check_refined(got, z, n, "oracle")
    r = got["ran1"]
    assert (r.idum, r.iy, r.mcall) == (int(z["ran1_after_idum"]), int(z["ran1_after_iy"]), int(z["ran1_after_mcall"]))
    assert np.array_equal(r.iv, z["ran1_after_iv"])
    # the case exercises what it is for: shared sets, weights that are not float32 values
    assert len(set(z["iref"].tolist())) < n["npairs"]
    assert not np.array_equal(z["cwt"].astype(f32).astype(np.float64), z["cwt"])
    if name == "ptgnsq_window":                         # the window rules are all in use
        assert n["nqmin"].min() > 1 and (n["szeros"] != 0).any() and (n["szeros"] == 0).any()
        assert (z["q"][1:] < n["qmin"]).any()
    if name == "ptgnsq_xray":                           # one X-ray set, one weighted by cwt
        assert z["xray"].tolist() == [1, 0] and (z["wq"][0, :, 1:] > 0).all()
        plain = oracle.ptgnsq_difference(z["data"], z["cwt"], z["qwind"], z["q"], n["nqmin"], n["nqmax"], n["szeros"],
                                         n["qmin"])
        assert not np.array_equal(plain[0], got["dt"][0]) and np.array_equal(plain[1], got["dt"][1])
