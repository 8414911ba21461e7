"""The host basis builders of generate_ep -- calc_pwrexpr_grad (epsr_standalone_rev3.py:5230)
and calc_gaussr_grad (:5046) in libepsr_gpu.so, computed on the CPU -- against the basis
matrix the reference built in each golden case of tests/golden/ep.npz, bit for bit."""

import numpy as np
import pytest

from epsr_python_translation_b200 import potential
from tests.goldens import GOLDEN, assert_bits_equal
from tests.test_ep_oracle import CASES


@pytest.mark.parametrize("name", CASES)
def test_basis_matches_reference(name):
    z = np.load(GOLDEN + "/ep.npz")
    npairs, npt, npt2, nterms, _ = (int(v) for v in z[f"{name}_dims"])
    gaussian, pdmin, pdstep, pdmax, psigma2, rho, rbroad = (np.float32(v) for v in z[f"{name}_basis"])
    expgr, ncfirst = potential.basis(npt2, nterms, z[f"{name}_x"], bool(gaussian), pdmin, pdstep, pdmax, psigma2, rho,
                                     rbroad)
    assert ncfirst == 0
    assert_bits_equal(expgr, z[f"{name}_expgr"], f"{name} expgr")
    assert np.count_nonzero(expgr) > expgr.size // 50   # the Gaussian basis is sparse


def test_basis_rejects_bad_arguments():
    from epsr_python_translation_b200._lib import EpsrGpuError
    with pytest.raises(EpsrGpuError):
        potential.basis(10, 5, np.linspace(0, 1, 11, dtype=np.float32), False, 1.01, 0.1, 12.0, 0.0, 0.1, 0.0)
