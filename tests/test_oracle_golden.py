"""Pin the C oracle (oracle/epsr_oracle.c) to the reference translation's own outputs.

Every fixture under tests/golden was produced by running the reference routines
(tests/golden/make_golden.py); ran1_reference.npz holds the reference's committed gfortran
bit patterns (tests/library/data/ran1_reference.txt).  All comparisons are bitwise.
"""

import os

import numpy as np
import pytest

from epsr_python_translation_b200.box import BoxArrays, Ran1State
from oracle import oracle
from tests import goldens
from tests.goldens import assert_bits_equal

f32 = np.float32


# ----------------------------------------------------------------------------- ran1
def test_ran1_gfortran_reference_blocks():
    z = np.load(goldens.GOLDEN + "/ran1_reference.npz")
    n = int(z["nblocks"])
    assert n == 7
    st = Ran1State()
    for k in range(n):
        head = str(z[f"block{k}_header"])
        if head.startswith("seed"):
            st = Ran1State(idum=int(head.split()[1]), iy=0, mcall=0, iv=np.zeros(32, np.int32))
        else:
            assert head == "continued"
        vals, st = oracle.ran1_fill(st, 1000)
        assert np.array_equal(vals.view(np.uint32), z[f"block{k}_bits"]), head
        state = z[f"block{k}_state"]
        assert [st.mcall, st.idum, st.iy] == [int(v) for v in state[:3]], head
        assert np.array_equal(st.iv, state[3:35].astype(np.int32)), head


@pytest.mark.parametrize("seed", [0, -1, -12345, -2147483647, 123, -987654321])
def test_ran1_stream_matches_reference(seed):
    z = np.load(goldens.GOLDEN + "/ran1_stream.npz")
    key = f"seed_{seed}".replace("-", "m")
    vals, st = oracle.ran1_fill(Ran1State(idum=seed), 3000)
    assert np.array_equal(vals.view(np.uint32), z[key].view(np.uint32))
    assert st.idum == int(z[key + "_after_idum"]) and st.iy == int(z[key + "_after_iy"])
    assert np.array_equal(st.iv, z[key + "_after_iv"])


# ----------------------------------------------------------------------------- cells + store
def _cells(z, box):
    return oracle.cell_list(box, int(z["in_nmolcell"]), f32(z["in_sepmax"]))


@pytest.mark.parametrize("case", goldens.CASES)
def test_cell_list_matches_reference(case):
    z = goldens.load(case)
    box = BoxArrays.from_golden(z)
    c = _cells(z, box)
    for k in ("ncelldiva", "ncelldivb", "ncelldivc", "ncell", "maxcellno", "ncellneighb"):
        assert c[k] == int(z["cell_" + k]), k
    start, flat = goldens.golden_cells_csr(z)
    assert np.array_equal(c["cell_start"], start)
    assert np.array_equal(c["cell_mols"], flat)
    assert np.array_equal(c["molcellno"], z["cell_molcellno"])
    for k in ("ia", "ib", "ic"):
        assert np.array_equal(c[k + "_off"], z[f"cell_{k}cellneighb"])
    assert c["nnbrefmax"] == int(z["fm_nnbrefmax"])


@pytest.mark.parametrize("case", goldens.CASES)
def test_fmolec1_store_matches_reference(case):
    z = goldens.load(case)
    box = BoxArrays.from_golden(z)
    c = _cells(z, box)
    st = oracle.fmolec1(box, c, z["in_eintra"])
    assert st["nergpair"] == int(z["fm_nergpair"])
    assert np.array_equal(st["nergpairm"], z["fm_nergpairm"])
    M = st["nnbrefmax"]
    ref_mol = z["fm_molergpair"]
    ref_ref = z["fm_ergpairref"]
    for im in range(box.nmol):
        k = st["nergpairm"][im]
        assert np.array_equal(st["molergpair"][im, :k], ref_mol[:k, im] - 1), im
        assert np.array_equal(st["ergpairref"][im, :k], ref_ref[:k, im]), im
    assert_bits_equal(st["ergpair"][: st["nergpair"]], z["fm_ergpair"], "ergpair")
    assert_bits_equal(st["ftest"], z["fm_ftest"], "ftest")
    assert_bits_equal(st["ftestb"], z["fm_ftestb"], "ftestb")


def test_slot_one_quirk_is_exercised():
    """Single-atom molecules have zero intra energy, so slot 1 holds a real neighbour whose
    energy en_change never includes (ergpairreference.py:103-118, molfit.py:839)."""
    z = goldens.load("silica")
    assert np.all(z["in_eintra"] == 0)
    z2 = goldens.load("c1_water")
    # rigid water in float32: most molecules have a tiny nonzero intra energy, some exactly 0
    assert np.any(z2["in_eintra"] != 0) and np.any(z2["in_eintra"] == 0)


# ----------------------------------------------------------------------------- molfit
def mc_params(z, box):
    nmt = box.nmoltype
    return dict(rejrate=f32(z["in_rejrate"]), stepr=f32(z["in_stepr"]), stepm=f32(z["in_stepm"]),
                wholerot=z["in_wholerot"].copy(), wholetrans=z["in_wholetrans"].copy(),
                internrot=np.zeros(nmt, f32), interntrans=np.zeros(nmt, f32), ireset=0,
                nstepreject=np.zeros(box.nmol, np.int32))


@pytest.mark.parametrize("case", goldens.CASES)
def test_molfit_cycles_match_reference(case):
    z = goldens.load(case)
    box = BoxArrays.from_golden(z)
    c = _cells(z, box)
    st = oracle.fmolec1(box, c, z["in_eintra"])
    mc = mc_params(z, box)
    ran1 = Ran1State.from_golden(z, "mf_ran1_before_")
    fadds = f32(0.0)
    for cyc in range(int(z["mf_cycles"])):
        p = f"mf{cyc}_"
        fadds, tr, ran1 = oracle.molfit(box, c, st, mc, ran1, fadds)
        assert tr["nmoves"] == z[p + "den"].shape[0]
        assert np.array_equal(tr["im"], z[p + "im"] - 1)
        assert_bits_equal(tr["den"], z[p + "den"], p + "den")
        assert_bits_equal(tr["cosv"], z[p + "cos"], p + "cos")
        for k in ("xa", "ya", "za", "xadd", "yadd", "zadd"):
            assert_bits_equal(getattr(box, k), z[p + k], p + k)
        n = st["nergpair"]
        assert_bits_equal(st["ergpair"][:n], z[p + "ergpair"], p + "ergpair")
        assert_bits_equal(mc["wholerot"], z[p + "wholerot"], p + "wholerot")
        assert_bits_equal(mc["wholetrans"], z[p + "wholetrans"], p + "wholetrans")
        nmt = box.nmoltype
        assert np.array_equal(mc["nwhole"].reshape(2, nmt), z[p + "nwhole"])
        assert np.array_equal(mc["nmovem"].reshape(2, nmt), z[p + "nmovem"])
        assert np.array_equal(mc["nstepreject"], z[p + "nstepreject"])
        assert_bits_equal(fadds, z[p + "fadds"], p + "fadds")
        assert ran1.idum == int(z[p + "ran1_after_idum"]) and ran1.iy == int(z[p + "ran1_after_iy"])
        assert np.array_equal(ran1.iv, z[p + "ran1_after_iv"])


# ----------------------------------------------------------------------------- atogen
def _final_coords(z, box):
    last = int(z["mf_cycles"]) - 1
    for k in ("xa", "ya", "za", "xadd", "yadd", "zadd"):
        setattr(box, k, z[f"mf{last}_{k}"].copy())


@pytest.mark.parametrize("case", goldens.CASES)
def test_atogen_matches_reference(case):
    z = goldens.load(case)
    box = BoxArrays.from_golden(z)
    _final_coords(z, box)
    ran1 = Ran1State.from_golden(z, "ag_ran1_before_")
    wav, potex, ngr, ran1 = oracle.atogen(box, int(z["ag_ngrsamples_in"]), ran1, z["ag_rminex"])
    assert ngr == int(z["ag_ngrsamples"])
    npt1 = box.npt1
    ref = z["ag_wav"]  # (2, npt1, npairs), iz 1..npt1
    mine = wav[:, :, 1:npt1 + 1].transpose(0, 2, 1)
    assert_bits_equal(mine, ref, "wav")
    assert_bits_equal(potex, z["ag_potex"], "potex")
    assert ran1.idum == int(z["ag_ran1_after_idum"]) and np.array_equal(ran1.iv, z["ag_ran1_after_iv"])


# ----------------------------------------------------------------------------- gensq / stog
def gensq_inputs(z, box):
    npt1 = box.npt1
    nq = int(z["gs_nq"])
    ld = box.npt + 1
    wav = np.zeros((2, box.npairs, ld), f32)
    wav[:, :, 1:npt1 + 1] = z["ag_wav"].transpose(0, 2, 1)
    F = z["gs_foqols"]            # (npt1+1, nq+1)  F[j, i]
    rows = np.ascontiguousarray(F.T)  # (nq+1, npt1+1)
    ycoh = z["gs_ycoh"][: npt1 + 1]
    return nq, npt1, wav, rows, ycoh


@pytest.mark.parametrize("case", ["c1_water", "mix_small"])
def test_gensq_matches_reference(case):
    z = goldens.load(case)
    box = BoxArrays.from_golden(z)
    nq, npt1, wav, rows, ycoh = gensq_inputs(z, box)
    out = oracle.gensq(nq, npt1, wav, rows, ycoh, box.n2extr, np.ones(box.ntype, f32))
    ref = z["gs_sofq"]  # (2, nq, npairs)
    assert_bits_equal(out[:, :, 1:].transpose(0, 2, 1), ref, "sofq")


@pytest.mark.parametrize("case", ["c1_water", "mix_small"])
def test_stog_matches_reference(case):
    z = goldens.load(case)
    q = z["gs_q"]
    nq = q.shape[0] - 1
    sofq = z["gs_sofq"][1]           # intermolecular (nq, npairs)
    sp = np.zeros((sofq.shape[1], nq + 1), f32)
    sp[:, 1:] = sofq.T
    r = np.zeros(z["sg_r"].shape[0] + 1, f32)
    r[1:] = z["sg_r"]
    g = oracle.stog(f32(z["sg_rho"]), q, sp, r, z["sg_nqmin"], z["sg_nqmax"], z["sg_xwt"])
    assert_bits_equal(g[:, 1:].T, z["sg_gofr"], "gofr")


# ----------------------------------------------------------------------------- fit_expansion
@pytest.mark.parametrize("run", [0, 1])
def test_fit_expansion_matches_reference(run):
    z = np.load(goldens.GOLDEN + "/fitexp.npz")
    p = f"fx{run}_"
    nterms, npt = int(z["fx_nterms"]), int(z["fx_npt"])
    wtold = np.zeros(nterms + 1, f32)
    wtold[1:] = z[p + "wtold_in"]
    ran1 = Ran1State.from_golden(z, p + "ran1_before_")
    res, ran1 = oracle.fit_expansion(z["fx_yin"], z["fx_expr"], wtold, f32(z["fx_stepr_in"]), 1, npt,
                                     int(z[p + "ncfirst"]), nterms, 1000, int(z["fx_nfreq"]), ran1)
    assert_bits_equal(res["wt"][1:], z[p + "wt"], "wt")
    assert_bits_equal(res["wtold"][1:], z[p + "wtold"], "wtold")
    assert_bits_equal(res["yout"][1:], z[p + "yout"], "yout")
    for k in ("stepr", "acceptr", "rejrat", "chisq"):
        assert_bits_equal(res[k], z[p + k], k)
    assert ran1.idum == int(z[p + "ran1_after_idum"]) and ran1.mcall == int(z[p + "ran1_after_mcall"])


def test_oracle_triclinic_minimage_matches_reference():
    """minimagec on non-cubic lattices (minimagec.py:13-45), the oracle against the
    reference's own results (tests/golden/triclinic.npz), bit for bit, including a cubic cell
    whose off-diagonal components are cos(90 deg) residues."""
    z = np.load(os.path.join(goldens.GOLDEN, "triclinic.npz"))
    for case in z["cases"]:
        box = goldens.point_box(z[f"{case}_lat6"], z[f"{case}_pts"])
        oracle.minimage_centres(box)
        got = np.stack([box.xadd, box.yadd, box.zadd], axis=1)
        goldens.assert_bits_equal(got, z[f"{case}_out"], str(case))
