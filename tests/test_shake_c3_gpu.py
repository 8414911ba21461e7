"""The intramolecular branch of molfit at full size -- configuration C3, 20,000 water
(60,000 atoms), every molecule moved -- and the mixture of C2 (DMSO: 45 atom pairs a molecule,
more than one warp's lanes) on the device against the C oracle on the same box: the
intramolecular energies, the pair store built from them, and one intramolecular cycle
(coordinates, stored energies, counts, step sizes, faddbs, ran1 state) bit for bit."""

import numpy as np
import pytest
import torch

from epsr_python_translation_b200.box import BoxArrays, Ran1State, trsteps
from oracle import oracle
from tests.goldens import assert_bits_equal

pytestmark = pytest.mark.gpu
f32 = np.float32


@pytest.mark.parametrize("config", ["c3_water", "c2_mixture"])
def test_intramolecular_cycle_full_size_matches_oracle(config):
    from epsr_python_translation_b200 import configs
    from epsr_python_translation_b200.device import DeviceBox
    from epsr_python_translation_b200.intra import IntraModel
    s = getattr(configs, config)(seed=1)
    m = configs.intra_model(s)
    ob = BoxArrays.from_system(s)
    d = DeviceBox(BoxArrays.from_system(s))
    model = IntraModel(d, **m)
    e_dev = model.en_mole_intra().cpu().numpy()
    e_ora = oracle.en_mole_intra_all(ob, m)
    assert_bits_equal(e_dev, e_ora, "en_mole_intra")
    d.cell_list(10, f32(ob.sepmax))
    oc = oracle.cell_list(ob, 10, f32(ob.sepmax))
    d.fmolec1(e_ora, strict=True)
    ost = oracle.fmolec1(ob, oc, e_ora)
    st = d.download_store()
    assert_bits_equal(st["ergpair"], ost["ergpair"][: ost["nergpair"]], "store")
    M = oc["nnbrefmax"]
    ost = dict(nnbrefmax=M, nergpair=ost["nergpair"], nergpairm=np.ascontiguousarray(ost["nergpairm"], np.int32),
               molergpair=np.ascontiguousarray(ost["molergpair"][:, :M], np.int32).reshape(-1),
               ergpairref=np.ascontiguousarray(ost["ergpairref"][:, :M], np.int32).reshape(-1),
               ergpair=np.array(ost["ergpair"][: ost["nergpair"]], f32))
    nmt = ob.nmoltype
    tmax, tmin = trsteps(ob.natomr)
    it0 = np.full(nmt, f32(0.02) / f32(ob.dmax), f32)
    if nmt > 1:
        it0[0] = 0.0                               # the trstepmin start for the first type
    rot, tra = np.full(nmt, f32(10.0 / 180.0), f32), np.full(nmt, f32(0.5) / f32(ob.dmax), f32)
    ran1 = Ran1State(idum=-11)
    d.mc_setup(rejrate=f32(0.75), stepr=f32(1.0), stepm=f32(1.0), wholerot=rot, wholetrans=tra,
               internrot=np.full(nmt, f32(0.01)), interntrans=it0, ran1=ran1, trstepmax=tmax, trstepmin=tmin,
               fadds=f32(0.5))
    fb = torch.tensor([-0.25], dtype=torch.float32, device="cuda")
    nmovei = model.molfit_shake(1.0, fb).cpu().numpy()
    mc = dict(rejrate=f32(0.75), ireset=0, wholerot=rot.copy(), wholetrans=tra.copy(),
              internrot=np.full(nmt, f32(0.01)), interntrans=it0.copy())
    fadds, faddbs, onmovei, _, ran1_after = oracle.molfit_shake(ob, ost, mc, m, 1.0, ran1, f32(0.5), f32(-0.25))
    assert np.array_equal(nmovei, onmovei), (nmovei, onmovei)
    assert onmovei[nmt:].sum() > 0                  # some moves were rejected
    co = d.download_coords()
    for k in ("xa", "ya", "za", "xadd", "yadd", "zadd"):
        assert_bits_equal(co[k], getattr(ob, k), k)
    assert_bits_equal(d.download_store()["ergpair"], ost["ergpair"], "store after the cycle")
    mcd = d.download_mc()
    for k in ("interntrans", "internrot", "wholerot", "wholetrans"):
        assert_bits_equal(mcd[k], mc[k], k)
    assert_bits_equal(np.array([mcd["fadds"], fb.cpu().numpy()[0]], f32), np.array([fadds, faddbs], f32), "fadds")
    r = mcd["ran1"]
    assert (r.idum, r.iy) == (ran1_after.idum, ran1_after.iy) and np.array_equal(r.iv, ran1_after.iv)
