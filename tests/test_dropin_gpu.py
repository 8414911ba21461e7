"""The drop-in layer on the device: the reference's call sequence of one iteration
(initialise_cellneighbourlist -> fmolec1 -> molfit cycles -> atogen -> gensq -> stog, and
fit_expansion), made through the installed routines on COMMON blocks filled from the
golden fixtures, reproduces the reference's COMMON state bit for bit (the MC chain with
the reference's cosines injected)."""

import numpy as np
import pytest

from epsr_python_translation_b200 import dropin
from epsr_python_translation_b200.box import BoxArrays
from oracle import oracle
from tests import fake_common, goldens
from tests.goldens import assert_bits_equal

pytestmark = pytest.mark.gpu
f32 = np.float32


def _setup(case, strict):
    z = goldens.load(case)
    calls = []
    mods = fake_common.routine_modules(z, calls)
    c = fake_common.common_from_golden(z)
    path = dropin.PairPath(c, mods, strict=strict).install(dropin.ROUTINES)
    return z, c, mods, path, calls


def _cells_and_store(z, c, mods):
    cc, cnl, erd = c.clustercom, c.cellneighbourlist, c.ergpairreference
    mods["cellneighbourlist"].initialise_cellneighbourlist(int(z["in_nmolcell"]), cc.xadd, cc.yadd, cc.zadd,
                                                          cc.nmol, f32(z["in_sepmax"]))
    for k in ("ncelldiva", "ncelldivb", "ncelldivc", "ncell", "maxcellno", "ncellneighb"):
        assert getattr(cnl, k) == int(z["cell_" + k]), k
    assert np.array_equal(cnl.nmolsincell[1:], z["cell_nmolsincell"])
    assert np.array_equal(cnl.molsincell[1:, 1:], z["cell_molsincell"])
    assert np.array_equal(cnl.molcellno[1:], z["cell_molcellno"])
    n = cnl.ncellneighb
    for k in ("iacellneighb", "ibcellneighb", "iccellneighb"):
        assert np.array_equal(getattr(cnl, k)[1:n + 1], z["cell_" + k]), k
    ierr, nth, ftest, ftestb, fteth, fcc = mods["ato_manipulation_rev4"].fmolec1(0, 0, f32(0), f32(0), f32(0),
                                                                                 f32(0))
    assert ierr == 0 and fteth == 0 and fcc == 0
    assert_bits_equal(ftest, z["fm_ftest"], "ftest")
    assert_bits_equal(ftestb, z["fm_ftestb"], "ftestb")
    assert erd.nnbrefmax == int(z["fm_nnbrefmax"]) and erd.nergpair == int(z["fm_nergpair"])
    assert np.array_equal(erd.nergpairm[1:], z["fm_nergpairm"])
    assert np.array_equal(erd.molergpair[1:, 1:], z["fm_molergpair"])
    assert np.array_equal(erd.ergpairref[1:, 1:], z["fm_ergpairref"])
    assert_bits_equal(erd.ergpair[1:erd.nergpair + 1], z["fm_ergpair"], "ergpair")


@pytest.mark.parametrize("case,strict", [("c1_water", True), ("mix_small", True), ("silica", True),
                                         ("mix_small", False)])
def test_dropin_iteration_matches_reference_common_state(case, strict):
    z, c, mods, path, calls = _setup(case, strict)
    _cells_and_store(z, c, mods)
    mc, cc, erd, r = c.molecom, c.clustercom, c.ergpairreference, c.ran1com
    nmt = int(cc.nmoltype)
    fake_common.set_ran1(c, z, "mf_ran1_before_")
    fadds, faddbs, nisum = f32(0), f32(0), 1
    for cyc in range(int(z["mf_cycles"])):
        p = f"mf{cyc}_"
        path.cos_override = z[p + "cos"]
        fadds, faddbs, nisum = mods["molfit"].molfit(fadds, faddbs, nisum, 100, 5, 0)
        assert nisum == int(z[p + "nisum"])
        if strict:
            assert_bits_equal(fadds, z[p + "fadds"], p + "fadds")
        else:
            assert abs(float(fadds) - float(z[p + "fadds"])) <= 1e-5 * max(1.0, abs(float(z[p + "fadds"])))
        for k, arr in (("xa", mc.xa), ("ya", mc.ya), ("za", mc.za), ("xadd", cc.xadd), ("yadd", cc.yadd),
                       ("zadd", cc.zadd)):
            assert_bits_equal(arr[1:], z[p + k], p + k)
        assert_bits_equal(erd.ergpair[1:erd.nergpair + 1], z[p + "ergpair"], p + "ergpair")
        assert_bits_equal(cc.wholerot[1:], z[p + "wholerot"], p + "wholerot")
        assert_bits_equal(cc.wholetrans[1:], z[p + "wholetrans"], p + "wholetrans")
        assert np.array_equal(cc.nwhole[1:3, 1:nmt + 1], z[p + "nwhole"])
        assert np.array_equal(cc.nmovem[1:3, 1:nmt + 1], z[p + "nmovem"])
        assert np.array_equal(cc.nstepreject[1:], z[p + "nstepreject"])
        assert (r.idum, r.iy, r.mcall) == (int(z[p + "ran1_after_idum"]), int(z[p + "ran1_after_iy"]),
                                           int(z[p + "ran1_after_mcall"]))
        assert np.array_equal(r.iv[1:33], z[p + "ran1_after_iv"])
    # atogen continues the same ran1 stream on the final coordinates
    npairs, npt1 = int(mc.npairs), int(c.epsr16.npt1)
    wav = fake_common.fa(2, c.epsr16.npt + 8, npairs)
    n = mods["ato_manipulation_rev4"].atogen(wav, int(z["ag_ngrsamples_in"]))
    assert n == int(z["ag_ngrsamples"])
    assert_bits_equal(wav[1:3, 1:npt1 + 1, 1:npairs + 1], z["ag_wav"], "wav")
    assert_bits_equal(c.potential_par.potex[1:], z["ag_potex"], "potex")
    assert (r.idum, r.mcall) == (int(z["ag_ran1_after_idum"]), int(z["ag_ran1_after_mcall"]))
    assert np.array_equal(r.iv[1:33], z["ag_ran1_after_iv"])
    if "gs_sofq" in z.files:
        nq = int(z["gs_nq"])
        q = fake_common.fa(nq + 4)
        q[:nq + 1] = z["gs_q"]
        sofq = fake_common.fa(2, nq + 4, npairs)
        c.epsr16.ycoh[:z["gs_ycoh"].shape[0]] = z["gs_ycoh"]
        mods["program"].gensq(nq, q, sofq, wav)
        assert_bits_equal(sofq[1:3, 1:nq + 1, 1:npairs + 1], z["gs_sofq"], "sofq")
        nr = npt1
        sq2 = fake_common.fa(nq, npairs)
        sq2[1:nq + 1, 1:] = sofq[2, 1:nq + 1, 1:npairs + 1]
        rr = fake_common.fa(nr)
        rr[1:] = z["sg_r"]
        gofr = fake_common.fa(nr, npairs)
        lo = np.zeros(npairs + 1, np.int32)
        hi = np.zeros(npairs + 1, np.int32)
        lo[1:], hi[1:] = z["sg_nqmin"], z["sg_nqmax"]
        xwt = fake_common.fa(npairs)
        xwt[1:] = z["sg_xwt"]
        mods["ato_manipulation_rev4"].stog(f32(z["sg_rho"]), q, sq2, rr, gofr, lo, hi, nr, npairs, nq, nr, npairs,
                                           xwt)
        # the layout conversion only: identical to the device call it wraps, whose sine is
        # tolerance-checked against the reference in test_gpu_parity
        from epsr_python_translation_b200 import transforms
        sp = np.zeros((npairs, nq + 1), f32)
        sp[:, 1:] = z["gs_sofq"][1].T
        r0 = np.zeros(nr + 1, f32)
        r0[1:] = z["sg_r"]
        want = transforms.stog(f32(z["sg_rho"]), z["gs_q"], sp, r0, z["sg_nqmin"], z["sg_nqmax"],
                               z["sg_xwt"]).cpu().numpy()
        assert_bits_equal(gofr[1:, 1:], want[:, 1:].T, "gofr")
    assert calls == []          # nothing fell back to the host routines


@pytest.mark.parametrize("run", [0, 1])
def test_dropin_fit_expansion_matches_reference(run):
    z = np.load(goldens.GOLDEN + "/fitexp.npz")
    p = f"fx{run}_"
    nterms, npt = int(z["fx_nterms"]), int(z["fx_npt"])
    c = fake_common.common_from_golden(goldens.load("c1_water"))
    fake_common.set_ran1(c, z, p + "ran1_before_")
    path = dropin.PairPath(c, {}, strict=True)
    wt, wtold, yout = np.zeros(nterms + 1, f32), np.zeros(nterms + 1, f32), np.zeros(npt + 1, f32)
    wtold[1:] = z[p + "wtold_in"]
    out = path.fit_expansion(z["fx_yin"], z["fx_expr"], yout, wt, wtold, f32(z["fx_stepr_in"]),
                             f32(z[p + "acceptr_in"]), f32(0), f32(0), 1, npt, int(z[p + "ncfirst"]), nterms, 1000,
                             int(z["fx_nfreq"]))
    assert_bits_equal(wt[1:], z[p + "wt"], "wt")
    assert_bits_equal(wtold[1:], z[p + "wtold"], "wtold")
    assert_bits_equal(yout[1:], z[p + "yout"], "yout")
    for v, k in zip(out, ("stepr", "acceptr", "rejrat", "chisq")):
        assert_bits_equal(v, z[p + k], k)
    r = c.ran1com
    assert (r.idum, r.mcall) == (int(z[p + "ran1_after_idum"]), int(z[p + "ran1_after_mcall"]))


def test_dropin_sees_host_changes_between_calls():
    """A coordinate the host moves between device calls is uploaded before the next one;
    a host-built cell list is refused."""
    z, c, mods, path, calls = _setup("mix_small", True)
    _cells_and_store(z, c, mods)
    cc = c.clustercom
    cc.xadd[1] = cc.xadd[1] + f32(0.01)
    e = mods["molfit"].en_mole_pair(1, 2)
    ob = BoxArrays.from_golden(z)
    ob.xadd[0] = cc.xadd[1]
    assert_bits_equal(e, oracle.en_mole_pair(ob, 0, 1), "en_mole_pair after a host move")
    c.cellneighbourlist.molcellno[1] += 1
    with pytest.raises(dropin.EpsrGpuError):
        mods["molfit"].molfit(f32(0), f32(0), 1, 100, 5, 0)


@pytest.mark.parametrize("case", ["c1_water", "mix_small", "silica"])
def test_dropin_press_matches_reference(case):
    """press through the installed routine, right after fmolec1 (the state the press golden
    was made in): energy, pressure and the per-file rescaling bit for bit."""
    from tests.test_press_oracle import press_case
    p = press_case(case)
    z, c, mods, path, calls = _setup(case, True)
    _cells_and_store(z, c, mods)
    c.clustercom.volume = p[case + "_volume"]
    c.epsr16.nfile = 1
    c.potential_par.wsum[1] = f32(1.0)
    energf, pressf = fake_common.fa(4), fake_common.fa(4)
    energf[1], pressf[1] = p[case + "_energf_in"], p[case + "_pressf_in"]
    energy, pressc, energabs, energthreeb, prthree = mods["ato_manipulation_rev4"].press(
        f32(0), f32(0), energf, pressf, f32(0), f32(0), f32(0))
    assert_bits_equal(energy, p[case + "_energy"], "energy")
    assert_bits_equal(pressc, p[case + "_pressc"], "pressc")
    assert_bits_equal(energf[1], p[case + "_energf"], "energf")
    assert_bits_equal(pressf[1], p[case + "_pressf"], "pressf")
    assert energabs == 0 and energthreeb == 0 and calls == []
