"""The fast molfit cycle's draws ahead (mc_spec.cu): the next cycle's ran1 values walked on a
second stream while a cycle runs.  A box run with them and a box run without them, from the
same state, stay identical bit for bit -- coordinates, stored energies, step sizes and the
ran1 stream -- over several cycles, also when another stage draws from the stream between
cycles (atogen here), where the values walked ahead must not be taken."""

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _box(seed):
    from epsr_python_translation_b200 import configs
    from epsr_python_translation_b200.box import BoxArrays, Ran1State, trsteps
    from epsr_python_translation_b200.device import DeviceBox
    wl = configs.make_workload("c2_mixture", ntimes=1)
    box = BoxArrays.from_system(wl.system)
    d = DeviceBox(box)
    d.cell_list(wl.nmolcell, box.sepmax)
    d.fmolec1(wl.eintra, strict=False)
    tmax, tmin = trsteps(box.natomr)
    d.mc_setup(rejrate=np.float32(0.75), stepr=1.0, stepm=1.0, wholerot=wl.wholerot, wholetrans=wl.wholetrans,
               ran1=Ran1State(idum=seed), trstepmax=tmax, trstepmin=tmin)
    return d, box


def _same(a, b):
    ca, cb = a.download_coords(), b.download_coords()
    for k in ca:
        assert np.array_equal(ca[k].view(np.uint32), cb[k].view(np.uint32)), k
    assert np.array_equal(a.m_ran1.cpu().numpy(), b.m_ran1.cpu().numpy())
    sa, sb = a.download_store(), b.download_store()
    assert np.array_equal(sa["ergpair"].view(np.uint32), sb["ergpair"].view(np.uint32))
    for k in ("m_wholerot", "m_wholetrans", "m_fadds"):
        assert np.array_equal(getattr(a, k).cpu().numpy().view(np.uint32), getattr(b, k).cpu().numpy().view(np.uint32)), k


def test_draws_ahead_leave_every_cycle_unchanged():
    a, _ = _box(-21)
    b, _ = _box(-21)
    assert b.draws_ahead(False) == 0
    for _ in range(5):
        a.molfit(strict=False)
        b.molfit(strict=False)
    torch.cuda.synchronize()
    a.check_status()
    b.check_status()
    _same(a, b)
    assert a.draws_ahead(True) == 4          # every cycle after the first took the values walked ahead
    assert int(b.m_ahead[2].item()) == 0


def test_draws_ahead_not_taken_after_another_stage_drew():
    a, box = _box(-33)
    b, _ = _box(-33)
    b.draws_ahead(False)
    for cyc in range(4):
        for d in (a, b):
            d.molfit(strict=False)
            if cyc % 2 == 0:     # atogen over 50 origins draws from the same stream
                d.atogen(50, d.m_ran1, np.full(box.npairs, -2.0, np.float32))
    torch.cuda.synchronize()
    _same(a, b)
    # cycles 1 and 3 follow an atogen call, cycle 2 follows cycle 1 directly
    assert a.draws_ahead(True) == 1
