"""The intramolecular branch of molfit (molfit.py:124-174, then :465-536) and en_mole_intra
(:1327) on the device through the C ABI (epsr_molfit_shake, epsr_en_mole_intra), against the
reference run on seeded systems (tests/golden/shake.npz), bit for bit over two cycles; the
pair store the cycles start from is built by the device cell list and fmolec1 from the
reference's intramolecular energies."""

import numpy as np
import pytest
import torch

from epsr_python_translation_b200.box import BoxArrays, Ran1State, trsteps
from tests.goldens import GOLDEN, assert_bits_equal
from tests.test_shake_oracle import CASES, Prefixed

pytestmark = pytest.mark.gpu
f32 = np.float32


def _setup(name):
    from epsr_python_translation_b200.device import DeviceBox
    from epsr_python_translation_b200.intra import IntraModel
    z = np.load(GOLDEN + "/shake.npz")
    p = Prefixed(z, name + "_")
    box = BoxArrays.from_golden(p)
    d = DeviceBox(box)
    d.cell_list(10, box.sepmax)
    d.fmolec1(p["eintra"], strict=True)
    sc = p["scal"]
    tmax, tmin = trsteps(box.natomr)
    d.mc_setup(rejrate=0.75, stepr=1.0, stepm=1.0, wholerot=p["wholerot_in"], wholetrans=p["wholetrans_in"],
               internrot=p["internrot_in"], interntrans=p["interntrans_in"], ran1=Ran1State.from_golden(p, "ran1_before_"),
               trstepmax=tmax, trstepmin=tmin, fadds=p["fadds_in"])
    model = IntraModel(d, nbond=p["nbond"], iabond=p["iabond"], tbond=p["tbond"], amassa=p["amassa"],
                       amassr=p["amassr"], xav=p["xav"], xav1=p["xav1"], stepcl=sc[0], sizefactor=sc[1], tempb=sc[2],
                       tempang=sc[3], simt=sc[4], refine_intra=bool(sc[5]), refine_intra_fac=sc[6])
    return p, box, d, model, f32(sc[7])


@pytest.mark.parametrize("name", CASES)
def test_en_mole_intra_device_matches_reference(name):
    p, box, d, model, _ = _setup(name)
    assert_bits_equal(model.en_mole_intra().cpu().numpy(), p["eintra"], f"{name} eintra")


@pytest.mark.parametrize("name", CASES)
def test_shake_cycle_device_matches_reference(name):
    p, box, d, model, stepmi = _setup(name)
    co = d.download_coords()
    for k in co:                                    # the cycles start where the reference's did
        assert_bits_equal(co[k], p["in_" + k], f"{name} start {k}")
    st = d.download_store()
    assert_bits_equal(st["ergpair"], p["in_ergpair"], f"{name} start store")
    faddbs = torch.tensor([float(p["faddbs_in"])], dtype=torch.float32, device="cuda")
    for c in range(int(p["cycles"])):
        q = f"c{c}_"
        nmovei = model.molfit_shake(stepmi, faddbs).cpu().numpy()
        co = d.download_coords()
        for k in co:
            assert_bits_equal(co[k], p[q + k], f"{name} cycle {c} {k}")
        assert_bits_equal(d.download_store()["ergpair"], p[q + "ergpair"], f"{name} cycle {c} ergpair")
        mc = d.download_mc()
        for k in ("interntrans", "internrot", "wholerot", "wholetrans"):
            assert_bits_equal(mc[k], p[q + k], f"{name} cycle {c} {k}")
        assert np.array_equal(nmovei, p[q + "nmovei"].reshape(-1)), (nmovei, p[q + "nmovei"])
        assert np.array_equal(mc["nwhole"], p[q + "nwhole"]) and np.array_equal(mc["nmovem"], p[q + "nmovem"])
        assert_bits_equal(np.array([mc["fadds"], faddbs.cpu().numpy()[0]], f32),
                          np.array([p[q + "fadds"], p[q + "faddbs"]], f32), f"{name} cycle {c} fadds, faddbs")
        r = mc["ran1"]
        assert (r.idum, r.iy) == (int(p[q + "ran1_after_idum"]), int(p[q + "ran1_after_iy"]))
        assert np.array_equal(r.iv, p[q + "ran1_after_iv"])


def test_shake_refuses_rotational_groups_before_any_change():
    from epsr_python_translation_b200._lib import EpsrGpuError
    from epsr_python_translation_b200.intra import IntraModel
    p, box, d, model, stepmi = _setup("mix")
    ngrot = np.zeros(box.nmol, np.int32)
    ngrot[3] = 1
    m2 = IntraModel(d, nbond=p["nbond"], iabond=p["iabond"], tbond=p["tbond"], amassa=p["amassa"], amassr=p["amassr"],
                    xav=p["xav"], xav1=p["xav1"], stepcl=p["scal"][0], simt=p["scal"][4], ngrot=ngrot)
    before = d.download_coords()
    r0 = d.m_ran1.cpu().numpy().copy()
    with pytest.raises(EpsrGpuError):
        m2.molfit_shake(stepmi, torch.zeros(1, device="cuda"))
    after = d.download_coords()
    for k in before:
        assert_bits_equal(after[k], before[k], k)
    assert np.array_equal(d.m_ran1.cpu().numpy(), r0)


class _Aliased(Prefixed):
    """The case's keys under the names the COMMON stand-ins read."""
    ALIAS = {"in_eintra": "eintra"}

    def __getitem__(self, k):
        return super().__getitem__(self.ALIAS.get(k, k))

    def __contains__(self, k):
        return super().__contains__(self.ALIAS.get(k, k))

    @property
    def files(self):
        return [k[len(self.p):] for k in self.z.files if k.startswith(self.p)]


@pytest.mark.parametrize("name", CASES)
def test_shake_dropin_matches_reference(name):
    """PairPath.fmolec1 (intramolecular energies on the device) and PairPath.molfit with
    nisum >= intra on COMMON stand-ins carrying the reference's molecom bond lists, masses and
    potential_par.xav tables: the COMMON state after each cycle equals the reference's, and no
    host routine ran."""
    from epsr_python_translation_b200 import dropin
    from tests import fake_common
    z = np.load(GOLDEN + "/shake.npz")
    p = _Aliased(z, name + "_")
    calls = []
    mods = fake_common.routine_modules(p, calls)
    c = fake_common.common_from_golden(p)
    mc, cc, pp, erd, r = c.molecom, c.clustercom, c.potential_par, c.ergpairreference, c.ran1com
    natom, nmol, ntype = mc.natom, cc.nmol, mc.ntype
    npairs, npt, nmt = mc.npairs, c.epsr16.npt, int(cc.nmoltype)
    fa = fake_common.fa
    iab = p["iabond"]
    mb = iab.shape[1]
    mc.nbond = fa(natom, dtype=np.int32)
    mc.nbond[1:] = p["nbond"]
    mc.iabond = fa(natom, mb, dtype=np.int32)
    mc.iabond[1:, 1:] = iab + 1
    mc.tbond = fa(natom, mb)
    mc.tbond[1:, 1:] = p["tbond"]
    mc.imageatom, mc.qtype = fa(natom, dtype=np.int32), fa(natom, dtype=np.int32)
    mc.amassa, mc.amassr = fa(ntype), fa(npairs)
    mc.amassa[1:], mc.amassr[1:] = p["amassa"], p["amassr"]
    sc = p["scal"]
    mc.sizefactor, mc.tempb, mc.tempangreq, mc.tempangwt = f32(sc[1]), f32(sc[2]), f32(sc[3]), f32(sc[3])
    mc.refine_intra, mc.refine_intra_fac, mc.stepmi = bool(sc[5]), f32(sc[6]), f32(sc[7])
    mpz = pp.xavs.shape[0] - 1
    pp.xav, pp.xav1 = fa(mpz, npairs), fa(mpz, npairs)
    pp.xav[: npt + 1, 1:], pp.xav1[: npt + 1, 1:] = p["xav"].T, p["xav1"].T
    cc.interntrans[1:], cc.internrot[1:] = p["interntrans_in"], p["internrot_in"]
    dropin.PairPath(c, mods, strict=True).install(dropin.ROUTINES)
    mods["cellneighbourlist"].initialise_cellneighbourlist(int(p["in_nmolcell"]), cc.xadd, cc.yadd, cc.zadd, nmol,
                                                          f32(p["in_sepmax"]))
    mods["ato_manipulation_rev4"].fmolec1(0, 0, f32(0), f32(0), f32(0), f32(0))
    assert_bits_equal(erd.ergpair[1:erd.nergpair + 1], p["in_ergpair"], "store before the cycles")
    fake_common.set_ran1(c, p, "ran1_before_")
    fadds, faddbs = f32(p["fadds_in"]), f32(p["faddbs_in"])
    for cyc in range(int(p["cycles"])):
        q = f"c{cyc}_"
        fadds, faddbs, nisum = mods["molfit"].molfit(fadds, faddbs, 1, 1, 5, 0)
        assert nisum == int(p[q + "nisum"])
        assert_bits_equal(np.array([fadds, faddbs], f32), np.array([p[q + "fadds"], p[q + "faddbs"]], f32),
                          q + "fadds, faddbs")
        for k, arr in (("xa", mc.xa), ("ya", mc.ya), ("za", mc.za), ("xadd", cc.xadd), ("yadd", cc.yadd),
                       ("zadd", cc.zadd)):
            assert_bits_equal(arr[1:], p[q + k], q + k)
        assert_bits_equal(erd.ergpair[1:erd.nergpair + 1], p[q + "ergpair"], q + "ergpair")
        for k in ("interntrans", "internrot", "wholerot", "wholetrans"):
            assert_bits_equal(getattr(cc, k)[1:], p[q + k], q + k)
        for k in ("nmovei", "nwhole", "nmovem"):
            assert np.array_equal(getattr(cc, k)[1:3, 1:nmt + 1], p[q + k]), k
        assert (r.idum, r.iy, r.mcall) == (int(p[q + "ran1_after_idum"]), int(p[q + "ran1_after_iy"]),
                                           int(p[q + "ran1_after_mcall"]))
    assert not [k for k in calls if k.startswith("host:")], calls
