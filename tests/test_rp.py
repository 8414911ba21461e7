"""The reference potential tables -- generate_mp (ato_manipulation_rev4.py:2816) and generate_rp
(epsr_standalone_rev3.py:5675-5873) in libepsr_gpu.so, computed on the host -- against the
reference run on seeded parameters (tests/golden/rp.npz, made by tests/golden/make_golden_rp.py),
bit for bit: every branch of chsph, Gaussians of either sign, gauss6pot's modified Morse, both
repulsive cores with and without a gradient limit, coul_intra and shared coefficient sets."""

import numpy as np
import pytest

from epsr_python_translation_b200 import potential
from tests.goldens import GOLDEN, assert_bits_equal

CASES = ["lj", "gauss", "morse"]


def tables(z, name):
    p = lambda k: z[f"{name}_{k}"]  # noqa: E731
    npairs, npt, npt2, ntype, nsets, maxg = (int(v) for v in p("dims"))
    power, ecore, dcore, sizefactor, refpotfac, expecf, gradlimit, harmonic, modmorse, coul_intra, cif = p("scal")
    pairs = p("pairs")
    return potential.reference_potential(
        p("x"), p("xstar"), p("wfac"), p("wfacc"), npt, npt2, pairs[:, 0], pairs[:, 1], p("iref"), p("qradius"),
        p("ecor"), p("qcor"), p("dcor"), p("coulfac"), p("pcoefex"), p("rminex"), power, ecore, dcore, sizefactor,
        refpotfac, expecf, gradlimit, bool(harmonic), bool(modmorse), bool(coul_intra), cif, p("npgauss"),
        p("wpgauss"), p("rpgauss"), p("hpgauss")), npt


@pytest.mark.parametrize("name", CASES)
def test_reference_potential_matches_reference(name):
    z = np.load(GOLDEN + "/rp.npz")
    got, npt = tables(z, name)
    for k in potential.RP_TABLES:
        assert_bits_equal(got[k][:, 1:], z[f"{name}_{k}"][:, 1:], f"{name} {k}")


def test_reference_potential_cases_cover_the_branches():
    z = np.load(GOLDEN + "/rp.npz")
    sc = {n: z[f"{n}_scal"] for n in CASES}
    assert sc["gauss"][7] == 1.0 and sc["lj"][7] == 0.0          # harmonic and exponential cores
    assert sc["morse"][8] == 1.0 and sc["gauss"][9] == 1.0        # modified Morse, coul_intra
    assert sc["lj"][6] == 0.0 and sc["morse"][6] > 0.0           # with and without a gradient limit
    assert (z["gauss_hpgauss"] < 0).any() and (z["gauss_hpgauss"] > 0).any()
    assert len(set(z["gauss_iref"].tolist())) < len(z["gauss_iref"])
    assert np.isfinite(z["lj_ecoul"][:, 1:]).all()


@pytest.mark.parametrize("name", CASES)
def test_reference_potential_dropin_matches_reference(name):
    """PairPath.generate_rp() on COMMON-style 1-based Fortran arrays (no device needed)."""
    from types import SimpleNamespace as NS
    from epsr_python_translation_b200 import dropin
    z = np.load(GOLDEN + "/rp.npz")
    p = lambda k: z[f"{name}_{k}"]  # noqa: E731
    npairs, npt, npt2, ntype, nsets, maxg = (int(v) for v in p("dims"))
    power, ecore, dcore, sizefactor, refpotfac, expecf, gradlimit, harmonic, modmorse, coul_intra, cif = p("scal")
    mpz, mp, mg = npt + 9, npairs + 3, maxg + 2
    fa = lambda *d, dt=np.float32: np.zeros(d, dt, order="F")  # noqa: E731
    x, xs, wf, wc = fa(mpz), fa(mpz), fa(mpz), fa(mpz)
    x[: npt + 1], xs[: npt + 1], wf[: npt + 1], wc[: npt + 1] = p("x"), p("xstar"), p("wfac"), p("wfacc")
    mc = NS(npairs=npairs, ntype=ntype, n1extr=fa(mp, dt=np.int32), n2extr=fa(mp, dt=np.int32), qradius=fa(ntype + 3),
            ecor=fa(mp), qcor=fa(mp), dcor=fa(mp), power=np.float32(power), ecore=np.float32(ecore),
            dcore=np.float32(dcore), sizefactor=np.float32(sizefactor), coul_intra=bool(coul_intra),
            coul_intra_fac=np.float32(cif))
    pairs = p("pairs")
    mc.n1extr[1: npairs + 1], mc.n2extr[1: npairs + 1] = pairs[:, 0] + 1, pairs[:, 1] + 1
    mc.qradius[1: ntype + 1] = p("qradius")
    mc.ecor[1: npairs + 1], mc.qcor[1: npairs + 1], mc.dcor[1: npairs + 1] = p("ecor"), p("qcor"), p("dcor")
    pp = NS(irefpcof=fa(mp, dt=np.int32), coulfac=fa(mp), pcoefex=fa(mp), rminex=fa(mp), rmaxex=fa(mp),
            npgauss=fa(mp, dt=np.int32), wpgauss=fa(mg, mp), rpgauss=fa(mg, mp), hpgauss=fa(mg, mp),
            addpotential="modmorse" if modmorse else "", harmonic=bool(harmonic), refpotfac=np.float32(refpotfac),
            wfac=wf, wfacc=wc, **{k: fa(mpz, mp) for k in potential.RP_TABLES})
    pp.irefpcof[1: npairs + 1] = p("iref") + 1
    for k in ("coulfac", "pcoefex", "rminex", "npgauss"):
        getattr(pp, k)[1: nsets + 1] = p(k)
    for k in ("wpgauss", "rpgauss", "hpgauss"):
        getattr(pp, k)[1: maxg + 1, 1: nsets + 1] = p(k).T
    common = NS(molecom=mc, potential_par=pp, epsr16=NS(x=x, xstar=xs, npt=npt, npt2=npt2),
                epsrinput_par=NS(expecf=np.float32(expecf), expecfpwr=np.float32(gradlimit)))
    path = dropin.PairPath(common, {})
    assert path.generate_rp() is None
    for k in potential.RP_TABLES:
        assert_bits_equal(getattr(pp, k)[1: npt + 1, 1: npairs + 1].T, z[f"{name}_{k}"][:, 1:], f"{name} {k}")
