"""The EP refinement that follows the fits (ptgnsq epsr_standalone_rev3.py:3948-3962, then
generate_ep(.false.) :4014) on the device: the coefficient increment against the oracle's
restatement, the packed tables, and the refinement stage of the iteration (Python and native
drivers) against the oracle on the inputs the stage saw."""

import numpy as np
import pytest
import torch

from tests.goldens import assert_bits_equal

pytestmark = pytest.mark.gpu
f32 = np.float32


def _dev(a, dtype=torch.float32):
    return torch.from_numpy(np.ascontiguousarray(a)).to(device="cuda", dtype=dtype)


def test_ep_update_matches_oracle_with_shared_sets():
    from epsr_python_translation_b200 import potential
    from oracle import oracle
    rng = np.random.default_rng(3)
    npairs, nsets, nterms, ndata, ldc = 57, 20, 116, 3, 121
    pc = (rng.standard_normal((nsets, ldc)) * 0.1).astype(f32)
    iref = rng.integers(0, nsets, npairs).astype(np.int32)
    efacp = rng.uniform(0.5, 1.5, nsets).astype(f32)
    cwtpot = rng.uniform(0.0, 1.0, (ndata, npairs))            # real*8, general doubles
    pw = (rng.standard_normal((ndata, nterms + 1)) * 0.3).astype(f32)
    d = _dev(pc)
    potential.ep_update(d, iref, _dev(efacp), _dev(cwtpot, torch.float64), _dev(pw), f32(0.2))
    want = oracle.ep_update(pc, iref, efacp, cwtpot, pw, f32(0.2))
    assert_bits_equal(d.cpu().numpy(), want, "pcoefp")
    assert not np.array_equal(want, pc)


def test_pack_tables():
    from epsr_python_translation_b200 import potential
    rng = np.random.default_rng(4)
    t = [rng.standard_normal((5, 301)).astype(f32) for _ in range(4)]
    tab = torch.zeros(4 * 5 * 301, device="cuda")
    potential.pack_tables(*(_dev(a) for a in t), tab)
    assert_bits_equal(tab.cpu().numpy().reshape(5, 301, 4), np.stack(t, axis=-1), "tab")


@pytest.mark.parametrize("native", [False, True])
def test_iteration_refinement_matches_oracle(native):
    """Step 3 of a C1 iteration (steps 2 and 3 from native code when native): the stage's
    coefficients, tables and packed tables equal the oracle's refinement of the inputs the
    stage saw (coefficients, tables and the fits' coefficients after step 2's stage)."""
    from epsr_python_translation_b200 import configs, potential
    from epsr_python_translation_b200.iteration import EpsrIteration
    from oracle import oracle
    wl = configs.make_workload("c1_water", ntimes=1)
    it = EpsrIteration(wl, strict=True, ran1_seed=-5, native=native)
    it.step()
    it.step()
    torch.cuda.synchronize()
    pc0 = it.ep_pcoefp.cpu().numpy().copy()
    tabs0 = {k: v.cpu().numpy().copy() for k, v in it.ep_tabs.items()}
    pw0 = it.ep_pwtold.cpu().numpy().copy()
    it.step()
    torch.cuda.synchronize()
    b, ep = it.box, wl.ep
    fits = it.pwtold.cpu().numpy()
    pc = oracle.ep_update(pc0, ep.iref, ep.efacp, wl.weights, fits, ep.potfac)
    expgr = oracle.calc_pwrexpr_grad(b.npt2, wl.nterms, ep.pdmin, ep.pdstep, ep.pdmax, ep.psigma2, ep.rho, b.x)
    tabs, pc, pw, pf, _, _ = oracle.generate_ep(b.npt, b.npt2, wl.nterms, expgr, pc, ep.iref, b.dmax, b.xstar, ep.wfac,
                                                b.ecoul, tabs0, pw0,
                                                np.array([ep.absolute_energy, ep.erequnit, ep.ereqstep, ep.potfacamp],
                                                         f32), ep.potfac, False)
    assert_bits_equal(it.ep_pcoefp.cpu().numpy(), pc, "pcoefp")
    assert_bits_equal(it.ep_pwtold.cpu().numpy()[1:], pw[1:], "pwtold")
    for k in potential.TABLES:
        assert_bits_equal(it.ep_tabs[k].cpu().numpy(), tabs[k], k)
    packed = np.stack([tabs["xavs"], tabs["xavs1"], b.ecoul, b.ecoul1], axis=-1)
    assert_bits_equal(it.d.tab.cpu().numpy().reshape(packed.shape), packed, "packed tables")
    assert not np.array_equal(pc, pc0)
