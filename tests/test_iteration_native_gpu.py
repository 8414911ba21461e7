"""The native iteration driver (epsr_iteration_step, csrc/iteration.cu) against the Python
driver of the same routines: after the first (sizing) step, every further step launched from
native code leaves the box in exactly the state the Python driver leaves it in."""

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("strict", [False, True])
def test_native_iteration_matches_python_driver(strict):
    from epsr_python_translation_b200 import configs
    from epsr_python_translation_b200.iteration import EpsrIteration
    wl = configs.make_workload("c1_water", ntimes=2)
    a = EpsrIteration(wl, strict=strict, ran1_seed=-5, native=True)
    b = EpsrIteration(wl, strict=strict, ran1_seed=-5, native=False)
    for _ in range(3):
        a.step()
        b.step()
    assert a._plan is not None          # steps 2 and 3 ran natively
    torch.cuda.synchronize()
    ca, cb = a.d.download_coords(), b.d.download_coords()
    for k in ca:
        assert np.array_equal(ca[k].view(np.uint32), cb[k].view(np.uint32)), k
    assert np.array_equal(a.ran1.cpu().numpy(), b.ran1.cpu().numpy())
    assert np.array_equal(a.pwtold.cpu().numpy().view(np.uint32), b.pwtold.cpu().numpy().view(np.uint32))
    assert np.array_equal(np.asarray(a.stepp).view(np.uint32), np.asarray(b.stepp).view(np.uint32))
    assert np.array_equal(a.sofq.cpu().numpy().view(np.uint32), b.sofq.cpu().numpy().view(np.uint32))
    assert np.array_equal(a.gofr.cpu().numpy().view(np.uint32), b.gofr.cpu().numpy().view(np.uint32))
    assert a.fit_trials == b.fit_trials
    assert a.pair_updates == b.pair_updates
    assert np.float32(a.energy) == np.float32(b.energy) and np.float32(a.pressc) == np.float32(b.pressc)
    assert tuple(map(np.float32, a.ftest)) == tuple(map(np.float32, b.ftest))
    assert a.nsum == b.nsum == 3
    assert a.ep is not None              # the workload refines its EP every iteration
    assert np.array_equal(a.ep_pcoefp.cpu().numpy().view(np.uint32), b.ep_pcoefp.cpu().numpy().view(np.uint32))
    assert np.array_equal(a.d.tab.cpu().numpy().view(np.uint32), b.d.tab.cpu().numpy().view(np.uint32))
    for k, v in {**a.sums_sq, **a.sums_gr}.items():
        w = {**b.sums_sq, **b.sums_gr}[k]
        assert np.array_equal(v.cpu().numpy().view(np.uint32), w.cpu().numpy().view(np.uint32)), k


def test_native_iteration_c2_runs_and_matches():
    """C2 (600 molecules, three data sets): two native steps after the sizing step agree with
    the Python driver on the coordinates and the ran1 stream."""
    from epsr_python_translation_b200 import configs
    from epsr_python_translation_b200.iteration import EpsrIteration
    wl = configs.make_workload("c2_mixture", ntimes=1)
    a = EpsrIteration(wl, ran1_seed=-9, native=True)
    b = EpsrIteration(wl, ran1_seed=-9, native=False)
    for _ in range(3):
        a.step()
        b.step()
    torch.cuda.synchronize()
    ca, cb = a.d.download_coords(), b.d.download_coords()
    for k in ca:
        assert np.array_equal(ca[k].view(np.uint32), cb[k].view(np.uint32)), k
    assert np.array_equal(a.ran1.cpu().numpy(), b.ran1.cpu().numpy())


@pytest.mark.parametrize("config", ["c1_water", "c2_mixture"])
def test_native_iteration_with_intramolecular_cycles_matches_python_driver(config):
    """Flexible molecules (intra = 2, three molfit cycles a step, so both branches run in
    every step and the counter carries over): the native driver's steps equal the Python
    driver's -- coordinates, ran1 stream, stored energies, faddbs and the counter."""
    from epsr_python_translation_b200 import configs
    from epsr_python_translation_b200.iteration import EpsrIteration
    wl = configs.make_workload(config, ntimes=3, intra=2)
    a = EpsrIteration(wl, ran1_seed=-7, native=True)
    b = EpsrIteration(wl, ran1_seed=-7, native=False)
    for _ in range(3):
        a.step()
        b.step()
    assert a._plan is not None
    torch.cuda.synchronize()
    ca, cb = a.d.download_coords(), b.d.download_coords()
    for k in ca:
        assert np.array_equal(ca[k].view(np.uint32), cb[k].view(np.uint32)), k
    assert np.array_equal(a.ran1.cpu().numpy(), b.ran1.cpu().numpy())
    assert a.nisum_mc == b.nisum_mc
    assert np.array_equal(a.faddbs.cpu().numpy().view(np.uint32), b.faddbs.cpu().numpy().view(np.uint32))
    assert float(b.faddbs.cpu()[0]) != 0.0                 # intramolecular moves were made
    sa, sb = a.d.download_store(), b.d.download_store()
    assert np.array_equal(sa["ergpair"].view(np.uint32), sb["ergpair"].view(np.uint32))
    assert np.array_equal(a._nmovei.cpu().numpy(), b._nmovei.cpu().numpy())


def test_native_iteration_with_methyl_rotations_matches_python_driver():
    """C2 with the DMSO methyl groups rotated internally in every second whole-molecule cycle
    (rotfreq 2): the native driver and the Python driver leave identical coordinates, stored
    energies, internal-rotation steps and ran1 streams, and rotations were tried and accepted."""
    from epsr_python_translation_b200 import configs
    from epsr_python_translation_b200.iteration import EpsrIteration
    wl = configs.make_workload("c2_mixture", ntimes=4, rotfreq=2)
    assert wl.rotfreq == 2
    a = EpsrIteration(wl, ran1_seed=-13, native=True)
    b = EpsrIteration(wl, ran1_seed=-13, native=False)
    for _ in range(3):
        a.step()
        b.step()
    torch.cuda.synchronize()
    ca, cb = a.d.download_coords(), b.d.download_coords()
    for k in ca:
        assert np.array_equal(ca[k].view(np.uint32), cb[k].view(np.uint32)), k
    assert np.array_equal(a.ran1.cpu().numpy(), b.ran1.cpu().numpy())
    assert np.array_equal(a.d.m_internrot.cpu().numpy(), b.d.m_internrot.cpu().numpy())
    assert np.array_equal(a.d.m_faddbs.cpu().numpy().view(np.uint32), b.d.m_faddbs.cpu().numpy().view(np.uint32))
    ni = b.d.m_ninter.cpu().numpy()
    assert ni[0] > 0 and ni[nmt_rej := wl.system.nmoltype] < ni[0]
    del nmt_rej


def test_native_iteration_with_rotations_in_intramolecular_cycles_matches_python_driver():
    """C2 with flexible molecules (intra = 2) and the DMSO methyl groups as rotational groups
    (rotfreq 2): the intramolecular cycles then rotate the groups after each molecule's atom
    moves (molfit.py:175-267, on the sequential kernel), the whole-molecule cycles every second
    time.  The native and the Python drivers leave identical coordinates, stored energies,
    counters, faddbs and ran1 streams, and both kinds of cycle ran."""
    from epsr_python_translation_b200 import configs
    from epsr_python_translation_b200.iteration import EpsrIteration
    wl = configs.make_workload("c2_mixture", ntimes=3, intra=2, rotfreq=2)
    assert wl.rotfreq == 2 and wl.intra == 2
    a = EpsrIteration(wl, ran1_seed=-17, native=True)
    b = EpsrIteration(wl, ran1_seed=-17, native=False)
    for _ in range(3):
        a.step()
        b.step()
    torch.cuda.synchronize()
    ca, cb = a.d.download_coords(), b.d.download_coords()
    for k in ca:
        assert np.array_equal(ca[k].view(np.uint32), cb[k].view(np.uint32)), k
    assert np.array_equal(a.ran1.cpu().numpy(), b.ran1.cpu().numpy())
    sa, sb = a.d.download_store(), b.d.download_store()
    assert np.array_equal(sa["ergpair"].view(np.uint32), sb["ergpair"].view(np.uint32))
    for x, y in ((a.faddbs, b.faddbs), (a.d.m_faddbs, b.d.m_faddbs), (a._nmovei, b._nmovei),
                 (a.d.m_ninter, b.d.m_ninter), (a.d.m_internrot, b.d.m_internrot)):
        assert np.array_equal(x.cpu().numpy().view(np.uint32), y.cpu().numpy().view(np.uint32))
    assert int(b._nmovei.cpu()[0]) > 0                     # atom moves were tried
    # rotations were tried: the DMSO type's rotation step was adapted away from its start (the
    # counters hold only the last cycle's, a whole-molecule cycle without rotations here)
    assert float(b.d.m_internrot.cpu()[0]) != float(wl.internrot[0])
    assert float(b.faddbs.cpu()[0]) != 0.0
