"""Configuration C3 at full size -- 20,000 rigid water (60,000 atoms, L = 84.3 A, g(r) bin
0.03 A, EP on, 2,552-molecule neighbour regions, 3.0 million stored pairs) -- on the device
against the C oracle on the same box: the cell list and the pair store bit for bit, one
strict molfit cycle with the oracle's cosines bit for bit (coordinates, stored energies,
ran1 state), and atogen over 1,000 sampled origins bit for bit."""

import numpy as np
import pytest

from epsr_python_translation_b200.box import BoxArrays, Ran1State, trsteps
from oracle import oracle
from tests.goldens import assert_bits_equal

pytestmark = pytest.mark.gpu
f32 = np.float32


@pytest.fixture(scope="module")
def c3():
    from epsr_python_translation_b200 import configs
    s = configs.c3_water(seed=1)
    return s, configs.intra_energies(s)


def test_c3_cells_store_molfit_atogen_match_oracle(c3):
    from epsr_python_translation_b200.device import DeviceBox
    s, eintra = c3
    ob = BoxArrays.from_system(s)
    d = DeviceBox(BoxArrays.from_system(s))
    # cell list and pair store
    d.cell_list(10, f32(ob.sepmax))
    oc = oracle.cell_list(ob, 10, f32(ob.sepmax))
    assert d.nnbrefmax == oc["nnbrefmax"]
    ft, fb = d.fmolec1(eintra, strict=True)
    ost = oracle.fmolec1(ob, oc, eintra)
    st = d.download_store()
    assert st["nergpair"] == ost["nergpair"]
    assert np.array_equal(st["nergpairm"], ost["nergpairm"])
    M = oc["nnbrefmax"]
    assert np.array_equal(st["molergpair"], ost["molergpair"][:, :M])
    assert np.array_equal(st["ergpairref"], ost["ergpairref"][:, :M])
    assert_bits_equal(st["ergpair"], ost["ergpair"][: ost["nergpair"]], "ergpair")
    assert_bits_equal(ft, ost["ftest"], "ftest")
    # one strict molfit cycle with the oracle's cosines
    nmt = ob.nmoltype
    tmax, tmin = trsteps(ob.natomr)
    rot, tra = np.full(nmt, f32(10.0 / 180.0), f32), np.full(nmt, f32(0.5) / f32(ob.dmax), f32)
    ran1 = Ran1State(idum=-3)
    d.mc_setup(rejrate=f32(0.75), stepr=f32(1.0), stepm=f32(1.0), wholerot=rot, wholetrans=tra,
               internrot=np.zeros(nmt, f32), interntrans=np.zeros(nmt, f32), ran1=ran1, trstepmax=tmax,
               trstepmin=tmin)
    omc = dict(rejrate=f32(0.75), stepr=f32(1.0), stepm=f32(1.0), wholerot=rot.copy(), wholetrans=tra.copy(),
               internrot=np.zeros(nmt, f32), interntrans=np.zeros(nmt, f32), ireset=0)
    _, tr, ran1_after = oracle.molfit(ob, oc, ost, omc, ran1)
    d.molfit(strict=True, cos_override=tr["cosv"])
    m = d.download_mc()
    assert np.array_equal(m["acc"], tr["acc"])
    co = d.download_coords()
    for k in ("xa", "ya", "za", "xadd", "yadd", "zadd"):
        assert_bits_equal(co[k], getattr(ob, k), k)
    assert_bits_equal(d.download_store()["ergpair"], ost["ergpair"][: ost["nergpair"]], "ergpair after molfit")
    assert m["ran1"].idum == ran1_after.idum and np.array_equal(m["ran1"].iv, ran1_after.iv)
    # atogen over 1,000 sampled origins from the moved configuration
    rminex = np.full(ob.npairs, -2.0, f32)
    t = d.ran1_tensor(Ran1State(idum=-4))
    ngr = d.atogen(1000, t, rminex)
    wav, potex, ongr, rst = oracle.atogen(ob, 1000, Ran1State(idum=-4), rminex)
    assert ngr == ongr
    dwav, dpotex = d.download_wav()
    assert_bits_equal(dwav, wav, "wav")
    assert_bits_equal(dpotex, potex, "potex")
    assert np.array_equal(t.cpu().numpy(), rst.as_array())


def test_c3_fast_store_and_speculative_cycle_match_oracle(c3):
    """The fast modes the iteration and the benchmark run, at full C3 size: the pair store
    built with fast sums is bit-identical to the oracle's (only ftest is summed in another
    order, within 1e-5 of the oracle's), and one speculative molfit cycle with the oracle's
    cosines takes the oracle's decisions -- every energy change within the tolerance of the
    FP64 change, every decision the Metropolis rule on the device's own change and draw, a
    different decision only at the threshold of its draw -- and, while the chains agree,
    leaves coordinates, stored energies and the ran1 state bit-identical."""
    from epsr_python_translation_b200.device import DeviceBox
    from tests.chain_check import check_decisions
    s, eintra = c3
    ob = BoxArrays.from_system(s)
    d = DeviceBox(BoxArrays.from_system(s))
    d.cell_list(10, f32(ob.sepmax))
    oc = oracle.cell_list(ob, 10, f32(ob.sepmax))
    ft, _ = d.fmolec1(eintra, strict=False)
    ost = oracle.fmolec1(ob, oc, eintra)
    st = d.download_store()
    assert st["nergpair"] == ost["nergpair"]
    assert_bits_equal(st["ergpair"], ost["ergpair"][: ost["nergpair"]], "ergpair (fast)")
    # ftest: the stored intermolecular energies (after the intramolecular block) over nmol; the
    # fast sum is a double sum, checked against the exact sum of the same float32 entries (the
    # reference's sequential float32 sum of 3 million terms is itself off by ~0.3%)
    e = ost["ergpair"][: ost["nergpair"]].astype(np.float64)
    nintra = int(np.count_nonzero(eintra))
    exact = e[nintra:].sum() / ob.nmol
    assert abs(float(ft) - exact) <= 1e-6 * np.abs(e[nintra:]).sum() / ob.nmol + 1e-6, (float(ft), exact)
    nmt = ob.nmoltype
    tmax, tmin = trsteps(ob.natomr)
    rot, tra = np.full(nmt, f32(10.0 / 180.0), f32), np.full(nmt, f32(0.5) / f32(ob.dmax), f32)
    ran1 = Ran1State(idum=-5)
    d.mc_setup(rejrate=f32(0.75), stepr=f32(1.0), stepm=f32(1.0), wholerot=rot, wholetrans=tra,
               internrot=np.zeros(nmt, f32), interntrans=np.zeros(nmt, f32), ran1=ran1, trstepmax=tmax,
               trstepmin=tmin)
    omc = dict(rejrate=f32(0.75), stepr=f32(1.0), stepm=f32(1.0), wholerot=rot.copy(), wholetrans=tra.copy(),
               internrot=np.zeros(nmt, f32), interntrans=np.zeros(nmt, f32), ireset=0)
    _, tr, ran1_after = oracle.molfit(ob, oc, ost, omc, ran1)
    d.molfit(strict=False, cos_override=tr["cosv"])
    d.check_status()
    m = d.download_mc()
    if check_decisions(m["den"], m["acc"], tr, ob.simt, 1e-5) == "parted":
        return
    co = d.download_coords()
    for k in ("xa", "ya", "za", "xadd", "yadd", "zadd"):
        assert_bits_equal(co[k], getattr(ob, k), k)
    assert_bits_equal(d.download_store()["ergpair"], ost["ergpair"][: ost["nergpair"]], "ergpair after molfit")
    assert m["ran1"].idum == ran1_after.idum and np.array_equal(m["ran1"].iv, ran1_after.iv)
