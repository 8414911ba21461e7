"""The C restatement of generate_ep (epsr_standalone_rev3.py:5876-6022: the empirical-potential
tables rebuilt from the EP coefficients) against the reference's own generate_ep run on seeded
state (tests/golden/ep.npz, made by tests/golden/make_golden_ep.py), bit for bit over two
consecutive calls, with the coefficient scaling, the potential factor and pwtold."""

import numpy as np
import pytest

from oracle import oracle
from tests.goldens import GOLDEN, assert_bits_equal

TABS = ("xavs", "xavs1", "xavtot", "xavtot1")
CASES = ["small", "noabs", "unit", "cap", "shrink", "shared", "gauss"]


def case_arrays(z, name):
    """The golden case in the device layout: tables (npairs, npt+1), coefficients (nsets, nterms+1)."""
    npairs, npt, npt2, nterms, ncalls = (int(v) for v in z[f"{name}_dims"])
    dmax, absolute_energy, erequnit, ereqstep, potfac, potfacamp = (np.float32(v) for v in z[f"{name}_scal"])
    tabs = {k: np.ascontiguousarray(z[f"{name}_in_{k}"].T) for k in TABS}
    calls = []
    for c in range(ncalls):
        want = {k: np.ascontiguousarray(z[f"{name}_c{c}_{k}"].T) for k in TABS}
        calls.append((want, np.ascontiguousarray(z[f"{name}_c{c}_pcoefp"].T), z[f"{name}_c{c}_pwtold"],
                      np.float32(z[f"{name}_c{c}_potfac"])))
    return dict(npairs=npairs, npt=npt, npt2=npt2, nterms=nterms, dmax=dmax, tabs=tabs,
                ecoul=np.ascontiguousarray(z[f"{name}_in_ecoul"].T), pcoefp=np.ascontiguousarray(z[f"{name}_in_pcoefp"].T),
                iref=z[f"{name}_iref"].astype(np.int32), expgr=z[f"{name}_expgr"], xstar=z[f"{name}_xstar"],
                wfac=z[f"{name}_wfac"], par=np.array([absolute_energy, erequnit, ereqstep, potfacamp], np.float32),
                potfac=potfac, calls=calls)


@pytest.mark.parametrize("name", CASES)
def test_generate_ep_oracle_matches_reference(name):
    z = np.load(GOLDEN + "/ep.npz")
    c = case_arrays(z, name)
    tabs, pc, pw, pf = c["tabs"], c["pcoefp"], np.zeros(c["nterms"] + 1, np.float32), c["potfac"]
    for i, (want, want_pc, want_pw, want_pf) in enumerate(c["calls"]):
        tabs, pc, pw, pf, energabs, pressfac = oracle.generate_ep(
            c["npt"], c["npt2"], c["nterms"], c["expgr"], pc, c["iref"], c["dmax"], c["xstar"], c["wfac"], c["ecoul"],
            tabs, pw, c["par"], pf, True)
        for k in TABS:
            assert_bits_equal(tabs[k], want[k], f"{name} call {i} {k}")
        assert_bits_equal(pc[:, 1:], want_pc[:, 1:], f"{name} call {i} pcoefp")
        assert_bits_equal(pw[1:], want_pw[1:], f"{name} call {i} pwtold")
        assert_bits_equal(np.float32(pf), want_pf, f"{name} call {i} potfac")


def test_generate_ep_golden_cases_cover_the_pressfac_rules():
    """The first call of each case: small and unit have an EP range below erequnit (pressfac =
    erequnit / range); cap has it above erequnit with no ereqstep (pressfac capped at 1); shrink
    has it above the absolute energy (pressfac = absolute energy / range < 1); noabs has no
    absolute energy (pressfac 0: the EP switched off)."""
    z = np.load(GOLDEN + "/ep.npz")
    seen = {}
    for name in CASES:
        c = case_arrays(z, name)
        _, _, _, _, energabs, pressfac = oracle.generate_ep(
            c["npt"], c["npt2"], c["nterms"], c["expgr"], c["pcoefp"], c["iref"], c["dmax"], c["xstar"], c["wfac"],
            c["ecoul"], c["tabs"], np.zeros(c["nterms"] + 1, np.float32), c["par"], c["potfac"], True)
        seen[name] = (float(energabs), float(pressfac))
    for name, erequnit in (("small", 0.5), ("unit", 20.0)):
        assert seen[name][0] < erequnit and seen[name][1] == pytest.approx(erequnit / seen[name][0], rel=1e-6)
    assert 0.1 < seen["cap"][0] < 3.0 and seen["cap"][1] == 1.0
    assert seen["shrink"][0] > 0.1 and seen["shrink"][1] == pytest.approx(0.1 / seen["shrink"][0], rel=1e-6)
    assert seen["noabs"] == (0.0, 0.0)
