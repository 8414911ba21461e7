"""generate_ep (epsr_standalone_rev3.py:5876-6022) on the device through the C ABI, against the
reference's own generate_ep run on seeded state (tests/golden/ep.npz) bit for bit over
consecutive calls, and against the oracle at a full-size table set (231 atom pairs sharing
150 coefficient sets, 1,000 r points, padded leading dimensions)."""

import numpy as np
import pytest
import torch

from tests.goldens import GOLDEN, assert_bits_equal
from tests.test_ep_oracle import CASES, TABS, case_arrays

pytestmark = pytest.mark.gpu
f32 = np.float32


def _dev(a):
    return torch.from_numpy(np.ascontiguousarray(a, f32)).cuda()


@pytest.mark.parametrize("name", CASES)
def test_generate_ep_device_matches_reference(name):
    from epsr_python_translation_b200 import potential
    z = np.load(GOLDEN + "/ep.npz")
    c = case_arrays(z, name)
    tabs = {k: _dev(v) for k, v in c["tabs"].items()}
    pc, pw, pf = _dev(c["pcoefp"]), torch.zeros(c["nterms"] + 1, device="cuda"), _dev([c["potfac"]])
    args = (c["npt"], c["npt2"], c["nterms"], _dev(c["expgr"]), pc, c["iref"], c["dmax"], _dev(c["xstar"]),
            _dev(c["wfac"]), _dev(c["ecoul"]), tabs, pw, *c["par"][:3], c["par"][3], pf)
    for i, (want, want_pc, want_pw, want_pf) in enumerate(c["calls"]):
        res = potential.generate_ep(*args, changepotfac=True).cpu().numpy()
        for k in TABS:
            assert_bits_equal(tabs[k].cpu().numpy(), want[k], f"{name} call {i} {k}")
        assert_bits_equal(pc.cpu().numpy()[:, 1:], want_pc[:, 1:], f"{name} call {i} pcoefp")
        assert_bits_equal(pw.cpu().numpy()[1:], want_pw[1:], f"{name} call {i} pwtold")
        assert_bits_equal(pf.cpu().numpy()[0], want_pf, f"{name} call {i} potfac")
        assert np.isfinite(res).all()


def _large_case(seed=11, npairs=231, nsets=150, nterms=116, pad=7, cpad=5):
    from epsr_python_translation_b200 import configs, potential
    rng = np.random.default_rng(seed)
    g = configs.make_rgrid(0.03, 30.0, 9.0, 12.0)
    npt, npt2 = g["npt"], g["npt2"]
    ld, ldc = npt + 1 + pad, nterms + 1 + cpad
    dmax = f32(60.0)
    x = np.zeros(ld, f32)
    x[: npt + 1] = g["x"]
    xstar = (x / dmax).astype(f32)
    expgr, _ = potential.basis(npt2, nterms, x, False, f32(1.0) + f32(0.1) / f32(9.0), 0.1, 12.0, 0.004, 0.1, 0.0)
    pc = np.zeros((nsets, ldc), f32)
    pc[:, 1] = rng.uniform(0.5, 1.5, nsets)
    pc[:, 2: nterms + 1] = rng.standard_normal((nsets, nterms - 1)) * 0.05
    pc[:, nterms + 1:] = 7.0                       # padding the call must not touch
    iref = rng.integers(0, nsets, npairs).astype(np.int32)
    wfac = np.ones(ld, f32)
    r = x[: npt + 1]
    wfac[: npt + 1] = np.where(r < 9.0, 1.0, np.where(r < 12.0, 0.5 * (1.0 + np.cos(np.pi * (r - 9.0) / 3.0)), 0.0))
    tabs = {k: (rng.standard_normal((npairs, ld)) * 0.2).astype(f32) for k in TABS}
    ecoul = (rng.standard_normal((npairs, ld)) * 0.2).astype(f32)
    return dict(npt=npt, npt2=npt2, nterms=nterms, expgr=expgr, pcoefp=pc, iref=iref, dmax=dmax, xstar=xstar,
                wfac=wfac, ecoul=ecoul, tabs=tabs, par=np.array([2.0, 0.5, 0.0, 0.5], f32), potfac=f32(0.3))


def test_generate_ep_full_size_matches_oracle():
    from epsr_python_translation_b200 import potential
    from oracle import oracle
    c = _large_case()
    tabs = {k: _dev(v) for k, v in c["tabs"].items()}
    pc, pw, pf = _dev(c["pcoefp"]), torch.zeros(c["nterms"] + 1, device="cuda"), _dev([c["potfac"]])
    want_t, want_pc, want_pw, want_pf = c["tabs"], c["pcoefp"], np.zeros(c["nterms"] + 1, f32), c["potfac"]
    for i in range(2):
        res = potential.generate_ep(c["npt"], c["npt2"], c["nterms"], _dev(c["expgr"]), pc, c["iref"], c["dmax"],
                                    _dev(c["xstar"]), _dev(c["wfac"]), _dev(c["ecoul"]), tabs, pw, *c["par"][:3],
                                    c["par"][3], pf).cpu().numpy()
        want_t, want_pc, want_pw, want_pf, energabs, pressfac = oracle.generate_ep(
            c["npt"], c["npt2"], c["nterms"], c["expgr"], want_pc, c["iref"], c["dmax"], c["xstar"], c["wfac"],
            c["ecoul"], want_t, want_pw, c["par"], want_pf, True)
        for k in TABS:
            assert_bits_equal(tabs[k].cpu().numpy(), want_t[k], f"call {i} {k}")
        assert_bits_equal(pc.cpu().numpy(), want_pc, f"call {i} pcoefp")
        assert_bits_equal(pw.cpu().numpy(), want_pw, f"call {i} pwtold")
        assert_bits_equal(pf.cpu().numpy()[0], want_pf, f"call {i} potfac")
        assert_bits_equal(res, np.array([energabs, pressfac], f32), f"call {i} energabs, pressfac")
    assert (pc.cpu().numpy()[:, c["nterms"] + 1:] == 7.0).all()


def test_generate_ep_refuses_a_bad_set_index_before_any_change():
    from epsr_python_translation_b200 import potential
    from epsr_python_translation_b200._lib import EpsrGpuError
    c = _large_case(npairs=4, nsets=3)
    tabs = {k: _dev(v) for k, v in c["tabs"].items()}
    pc = _dev(c["pcoefp"])
    bad = np.array([0, 1, 3, 2], np.int32)
    with pytest.raises(EpsrGpuError):
        potential.generate_ep(c["npt"], c["npt2"], c["nterms"], _dev(c["expgr"]), pc, bad, c["dmax"], _dev(c["xstar"]),
                              _dev(c["wfac"]), _dev(c["ecoul"]), tabs, torch.zeros(c["nterms"] + 1, device="cuda"),
                              *c["par"][:3], c["par"][3], _dev([c["potfac"]]))
    torch.cuda.synchronize()
    for k in TABS:
        assert_bits_equal(tabs[k].cpu().numpy(), c["tabs"][k], k)
    assert_bits_equal(pc.cpu().numpy(), c["pcoefp"], "pcoefp")


@pytest.mark.parametrize("name", ["shared", "gauss"])
def test_generate_ep_dropin_matches_reference(name):
    """PairPath.generate_ep(changepotfac) on COMMON-style 1-based Fortran arrays, the basis
    built by the library's host builder from the basis parameters."""
    from types import SimpleNamespace as NS
    from epsr_python_translation_b200 import dropin
    z = np.load(GOLDEN + "/ep.npz")
    c = case_arrays(z, name)
    npairs, npt, npt2, nterms = c["npairs"], c["npt"], c["npt2"], c["nterms"]
    gaussian, pdmin, pdstep, pdmax, psigma2, rho, rbroad = (f32(v) for v in z[f"{name}_basis"])
    nsets = int(c["iref"].max()) + 1
    mpz, mcoeff, mpairs = npt + 9, nterms + 4, npairs + 2

    def fa(*dims):
        return np.zeros(dims, f32, order="F")
    pp = NS(ncoeffp=nterms, npairspcof=nsets, irefpcof=np.zeros(mpairs, np.int32), pcoefp=fa(mcoeff, mpairs),
            pwtold=fa(mcoeff), expgr=np.zeros(npt2 * nterms + 50, f32), wfac=fa(mpz), ecoul=fa(mpz, mpairs),
            gaussian=bool(gaussian), pdmin=pdmin, pdstep=pdstep, pdmax=pdmax, psigma2=psigma2,
            absolute_energy=c["par"][0], erequnit=c["par"][1], ereqstep=c["par"][2], potfacamp=c["par"][3],
            potfac=c["potfac"])
    pp.irefpcof[1: npairs + 1] = c["iref"] + 1
    pp.pcoefp[: nterms + 1, 1: nsets + 1] = c["pcoefp"].T
    pp.wfac[: npt + 1] = c["wfac"]
    pp.ecoul[: npt + 1, 1: npairs + 1] = c["ecoul"].T
    for k in TABS:
        setattr(pp, k, fa(mpz, mpairs))
        getattr(pp, k)[: npt + 1, 1: npairs + 1] = c["tabs"][k].T
    x = np.zeros(mpz, f32)
    x[: npt + 1] = z[f"{name}_x"]
    xstar = np.zeros(mpz, f32)
    xstar[: npt + 1] = c["xstar"]
    common = NS(potential_par=pp, epsr16=NS(npt=npt, npt2=npt2, x=x, xstar=xstar, rho=rho),
                molecom=NS(npairs=npairs), clustercom=NS(dmax=c["dmax"]), epsrinput_par=NS(rbroad=rbroad))
    path = dropin.PairPath(common, {})
    for i, (want, want_pc, want_pw, want_pf) in enumerate(c["calls"]):
        assert path.generate_ep(True) is None
        for k in TABS:
            assert_bits_equal(getattr(pp, k)[: npt + 1, 1: npairs + 1], want[k].T, f"call {i} {k}")
        assert_bits_equal(pp.pcoefp[1: nterms + 1, 1: nsets + 1], want_pc[:, 1:].T, f"call {i} pcoefp")
        assert_bits_equal(pp.pwtold[1: nterms + 1], want_pw[1:], f"call {i} pwtold")
        assert_bits_equal(np.float32(pp.potfac), want_pf, f"call {i} potfac")
        assert_bits_equal(pp.expgr[1: npt2 * nterms + 1], z[f"{name}_expgr"], f"call {i} expgr")
