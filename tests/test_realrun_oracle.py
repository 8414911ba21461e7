"""The oracle against the reference's own epsr loop on its shipped run folder (EPSR-test: 200
DMSO + 400 water, the DMSO methyl groups as ROT groups, the run folder's potentials and
intramolecular model), tests/golden/realrun.npz made by tests/golden/make_golden_realrun.py:
the loop's first molfit call (the intramolecular cycle: atom moves, then the methyl rotations
tested with the intermolecular change, molfit.py:124-267), its second (a whole-molecule
cycle, :268-448) and its sixth (a whole-molecule cycle with the internal rotations of the
methyl groups, :295-360, after the first potential refinement) replayed from the state the
loop held at each call, bit for bit -- coordinates, stored energies, step sizes, counters,
fadds/faddbs and the ran1 stream; the loop's first cell list; the pair store the loop's fmolec1
had just built before
each of them, with its ftest and ftestb; and the refinement between the fifth and sixth calls:
its first atogen (histograms, potex, the ran1 stream), press (energy and pressure), gensq
(at every 20th Q point), the running sums sumsq and sumgr, fit_expansion (coefficients, fitted curve, step, rates, chi^2,
the ran1 stream) and the generate_ep on the fitted coefficients (tables, coefficients,
weights, potfac)."""

import os

import numpy as np
import pytest

from epsr_python_translation_b200.box import BoxArrays, Ran1State
from oracle import oracle
from tests.goldens import GOLDEN, assert_bits_equal

f32 = np.float32
PATH = os.path.join(GOLDEN, "realrun.npz")


def _box(z, q):
    kw = {}
    for k in BoxArrays.__dataclass_fields__:
        v = z[q + "box_" + k]
        kw[k] = v if v.ndim else v.item()
    return BoxArrays(**kw)


def _store(z, q):
    M, n = int(z[q + "st_nnbrefmax"]), int(z[q + "st_nergpair"])
    return dict(nnbrefmax=M, nergpair=n, nergpairm=np.array(z[q + "st_nergpairm"], np.int32),
                molergpair=np.ascontiguousarray(z[q + "st_molergpair"], np.int32).reshape(-1),
                ergpairref=np.ascontiguousarray(z[q + "st_ergpairref"], np.int32).reshape(-1),
                ergpair=np.array(z[q + "st_ergpair"], f32))


def _call(z, q):
    """The box, store, cells, MC parameters and intramolecular model of captured call q."""
    box = _box(z, q)
    st = _store(z, q)
    M = st["nnbrefmax"]
    cells = oracle.cells_from_arrays(z[q + "cl_dims"], z[q + "cl_cell_start"], z[q + "cl_cell_mols"],
                                     z[q + "cl_molcellno"], z[q + "cl_offsets"], M)
    par = z[q + "par"]
    mc = dict(rejrate=f32(par[0]), stepr=f32(par[1]), stepm=f32(par[2]), ireset=int(z[q + "args_int"][3]),
              wholerot=np.array(z[q + "wholerot"], f32), wholetrans=np.array(z[q + "wholetrans"], f32),
              internrot=np.array(z[q + "internrot"], f32), interntrans=np.array(z[q + "interntrans"], f32),
              ngrot=np.array(z[q + "ngrot"], np.int32), nstepreject=np.array(z[q + "nstepreject"], np.int32))
    sc = z[q + "in_scal"]
    model = dict(nbond=z[q + "in_nbond"], iabond=z[q + "in_iabond"], tbond=z[q + "in_tbond"],
                 imageatom=z[q + "in_imageatom"], qtype=z[q + "in_qtype"], amassa=z[q + "in_amassa"],
                 amassr=z[q + "in_amassr"], xav=z[q + "in_xav"], xav1=z[q + "in_xav1"], stepcl=sc[0], sizefactor=sc[1],
                 tempb=sc[2], tempang=sc[3], simt=sc[4], refine_intra=bool(sc[5]), refine_intra_fac=sc[6],
                 ngrot=z[q + "ngrot"])
    rot = dict(model=model, nrf=z[q + "rot_nrf"], nrl=z[q + "rot_nrl"], axis=z[q + "rot_axis"].reshape(-1),
               first=z[q + "rot_first"], last=z[q + "rot_last"], atoms=z[q + "rot_atoms"], stepri=f32(par[3]),
               rotcycle=1)
    return box, st, cells, mc, rot


def _check_after(z, q, box, st, mc, fadds, faddbs, ran1, ninter=None, nmovei=None):
    for k in ("xa", "ya", "za", "xadd", "yadd", "zadd"):
        assert_bits_equal(getattr(box, k), z[q + "after_" + k], q + k)
    assert_bits_equal(st["ergpair"], z[q + "after_ergpair"], q + "ergpair")
    for k in ("wholerot", "wholetrans", "internrot", "interntrans"):
        assert_bits_equal(mc[k], z[q + "after_" + k], q + k)
    assert np.array_equal(mc["nwhole"], z[q + "after_nwhole"].reshape(-1))
    assert np.array_equal(mc["nmovem"], z[q + "after_nmovem"].reshape(-1))
    if ninter is not None:
        assert np.array_equal(ninter, z[q + "after_ninter"].reshape(-1))
    if nmovei is not None:
        assert np.array_equal(nmovei, z[q + "after_nmovei"].reshape(-1))
    assert np.array_equal(mc["nstepreject"], z[q + "after_nstepreject"])
    assert_bits_equal(np.array([fadds, faddbs], f32), z[q + "result"], q + "fadds, faddbs")
    assert (ran1.idum, ran1.iy, ran1.mcall) == (int(z[q + "ran1_after_idum"]), int(z[q + "ran1_after_iy"]),
                                                 int(z[q + "ran1_after_mcall"]))
    assert np.array_equal(ran1.iv, z[q + "ran1_after_iv"])


@pytest.mark.skipif(not os.path.exists(PATH), reason="fixture absent")
def test_realrun_intramolecular_cycle_with_rotations_oracle_matches_reference():
    z = np.load(PATH)
    q = "k0_"
    nisum, intra = (int(v) for v in z[q + "args_int"][:2])
    assert nisum >= intra                                   # the loop's first call: the intramolecular branch
    box, st, _, mc, rot = _call(z, q)
    assert int(np.max(mc["ngrot"])) > 0
    fadds, faddbs = (f32(v) for v in z[q + "args"])
    fadds, faddbs, nmovei, ninter, _, ran1, cosv = oracle.molfit_shake_rot(
        box, st, mc, rot, f32(z[q + "par"][4]), Ran1State.from_golden(z, q + "ran1_before_"),
        fadds, faddbs, f32(z[q + "ergold1"]))
    assert_bits_equal(cosv, z[q + "cos"], "rotati cosines")
    _check_after(z, q, box, st, mc, fadds, faddbs, ran1, ninter=ninter, nmovei=nmovei)
    assert ninter[0] > 0 and nmovei.sum() > 0


@pytest.mark.skipif(not os.path.exists(PATH), reason="fixture absent")
def test_realrun_whole_molecule_cycle_oracle_matches_reference():
    z = np.load(PATH)
    q = "k1_"
    box, st, cells, mc, _ = _call(z, q)
    fadds = f32(z[q + "args"][0])
    fadds, tr, ran1 = oracle.molfit(box, cells, st, mc, Ran1State.from_golden(z, q + "ran1_before_"), fadds)
    assert_bits_equal(tr["cosv"], z[q + "cos"], "rotatm cosines")
    # no rotation this cycle: faddbs is the argument, unchanged by the oracle's whole-molecule cycle
    _check_after(z, q, box, st, mc, fadds, f32(z[q + "args"][1]) + f32(0.0) / f32(box.nmol), ran1)


@pytest.mark.skipif(not os.path.exists(PATH), reason="fixture absent")
def test_realrun_whole_molecule_cycle_with_rotations_oracle_matches_reference():
    z = np.load(PATH)
    q = "k2_"
    nisum, intra, rotfreq = (int(v) for v in z[q + "args_int"][:3])
    assert nisum < intra and nisum % rotfreq == 0          # a rotation cycle of the whole-molecule branch
    box, st, cells, mc, rot = _call(z, q)
    fadds, faddbs = (f32(v) for v in z[q + "args"])
    rot["faddbs"] = faddbs
    fadds, tr, ran1 = oracle.molfit(box, cells, st, mc, Ran1State.from_golden(z, q + "ran1_before_"), fadds, rot=rot)
    assert_bits_equal(tr["cosv"], z[q + "cos"], "rotati and rotatm cosines")
    _check_after(z, q, box, st, mc, fadds, tr["faddbs"], ran1, ninter=tr["ninter"])
    assert tr["ninter"][0] > 0


@pytest.mark.skipif(not os.path.exists(PATH), reason="fixture absent")
@pytest.mark.parametrize("q", ["k0_", "k1_", "k2_"])
def test_realrun_pair_store_oracle_matches_reference(q):
    """Each captured call follows the loop's fmolec1 (epsr_standalone_rev3.py:1280 at the start
    of an iteration, :1343 after the intramolecular cycle): the oracle's en_mole_intra and
    fmolec1 on the captured coordinates and cell list give the captured store (every used slot
    of molergpair and ergpairref, nergpairm, the stored energies) and the ftest, ftestb the loop
    handed to molfit, bit for bit."""
    z = np.load(PATH)
    box, st, cells, _, rot = _call(z, q)
    eintra = oracle.en_mole_intra_all(box, rot["model"])
    got = oracle.fmolec1(box, cells, eintra)
    assert got["nnbrefmax"] == st["nnbrefmax"] and got["nergpair"] == st["nergpair"]
    nm = st["nergpairm"]
    assert np.array_equal(got["nergpairm"], nm)
    M = st["nnbrefmax"]
    used = np.arange(M)[None, :] < nm[:, None]
    for k in ("molergpair", "ergpairref"):
        assert np.array_equal(got[k][used], st[k].reshape(-1, M)[used]), k
    assert_bits_equal(got["ergpair"][: st["nergpair"]], st["ergpair"], q + "ergpair")
    assert_bits_equal(np.array([got["ftest"], got["ftestb"]], f32), z[q + "args"], q + "ftest, ftestb")


@pytest.mark.skipif(not os.path.exists(PATH), reason="fixture absent")
def test_realrun_atogen_oracle_matches_reference():
    """The refinement's atogen (ato_manipulation_rev4.py:3640) as the loop called it: the
    intra- and intermolecular histograms, potex, the returned count and the ran1 stream."""
    z = np.load(PATH)
    box = _box(z, "ag_")
    wav, potex, n, ran1 = oracle.atogen(box, int(z["ag_ngrsamples"]), Ran1State.from_golden(z, "ag_ran1_before_"),
                                        z["ag_rminex"], z["ag_ycoh"], f32(z["ag_sizefactor"]))
    ref = z["ag_wav"]
    npt1 = ref.shape[1]
    assert_bits_equal(wav[:, :, 1:npt1 + 1].transpose(0, 2, 1), ref, "wav")
    assert_bits_equal(potex, z["ag_potex"], "potex")
    assert n == int(z["ag_result"])
    assert (ran1.idum, ran1.iy, ran1.mcall) == (int(z["ag_ran1_after_idum"]), int(z["ag_ran1_after_iy"]),
                                                 int(z["ag_ran1_after_mcall"]))
    assert np.array_equal(ran1.iv, z["ag_ran1_after_iv"])
    assert float(np.abs(ref[1]).sum()) > 0


@pytest.mark.skipif(not os.path.exists(PATH), reason="fixture absent")
def test_realrun_press_oracle_matches_reference():
    """The refinement's press (ato_manipulation_rev4.py:3903) as the loop called it, on the
    store the loop held: the energy per molecule and the pressure it returned."""
    z = np.load(PATH)
    box, st = _box(z, "pr_"), _store(z, "pr_")
    npt1, simt, volume = z["pr_scal"]
    r = oracle.press(box, st, int(npt1), f32(simt), f32(volume))
    assert_bits_equal(np.array([r["energy"], r["pressc"]], f32), z["pr_result"], "energy, pressure")


@pytest.mark.skipif(not os.path.exists(PATH), reason="fixture absent")
def test_realrun_fit_expansion_oracle_matches_reference():
    """The refinement's first fit_expansion (epsr_standalone_rev3.py:4806, from ptgnsq :3936) as
    the loop called it: coefficients, the fitted curve, step, acceptance, rejection ratio, chi^2
    and the ran1 stream."""
    z = np.load(PATH)
    nmin, npt, ncfirst, nterms, nits, nfreq = (int(v) for v in z["fx_int"])
    stepr, acceptr, rejrat, chisqnew = (f32(v) for v in z["fx_scal_in"])
    res, ran1 = oracle.fit_expansion(z["fx_yin"], z["fx_expr"], z["fx_wtold_in"], stepr, nmin, npt, ncfirst, nterms,
                                     nits, nfreq, Ran1State.from_golden(z, "fx_ran1_before_"), acceptr=acceptr,
                                     rejrat=rejrat, chisqnew=chisqnew)
    for k in ("wt", "wtold"):
        assert_bits_equal(res[k][1:], z["fx_" + k][1:], k)
    assert_bits_equal(res["yout"][1:], z["fx_yout"][1:], "yout")
    assert_bits_equal(np.array([res["stepr"], res["acceptr"], res["rejrat"], res["chisq"]], f32), z["fx_result"],
                      "stepr, acceptr, rejrat, chisq")
    assert (ran1.idum, ran1.iy, ran1.mcall) == (int(z["fx_ran1_after_idum"]), int(z["fx_ran1_after_iy"]),
                                                 int(z["fx_ran1_after_mcall"]))
    assert np.array_equal(ran1.iv, z["fx_ran1_after_iv"])


@pytest.mark.skipif(not os.path.exists(PATH), reason="fixture absent")
def test_realrun_generate_ep_oracle_matches_reference():
    """The refinement's generate_ep (epsr_standalone_rev3.py:5876, from ptgnsq :4014) on the
    coefficients the fits produced, from the basis the reference built: the four tables, the
    scaled coefficients, the weights and potfac."""
    z = np.load(PATH)
    npt, npt2, nterms, change = (int(v) for v in z["ge_int"])
    dmax, absolute_energy, erequnit, ereqstep, potfacamp, potfac = (f32(v) for v in z["ge_scal"])
    tabs = {k: z["ge_" + k + "_in"] for k in ("xavs", "xavs1", "xavtot", "xavtot1")}
    out, pc, pw, pf, _, _ = oracle.generate_ep(npt, npt2, nterms, z["ge_expgr"], z["ge_pcoefp_in"], z["ge_iref"], dmax,
                                               z["ge_xstar"], z["ge_wfac"], z["ge_ecoul"], tabs, z["ge_pwtold_in"],
                                               np.array([absolute_energy, erequnit, ereqstep, potfacamp], f32),
                                               potfac, bool(change))
    for k in tabs:
        assert_bits_equal(out[k], z["ge_" + k], k)
    assert_bits_equal(pc[:, : nterms + 1], z["ge_pcoefp"], "pcoefp")
    assert_bits_equal(pw, z["ge_pwtold"], "pwtold")
    assert_bits_equal(np.array([pf], f32), np.array([z["ge_potfac"]], f32), "potfac")
    assert float(np.abs(z["ge_pcoefp_in"][:, 2:]).max()) > 0      # the fits moved the coefficients


@pytest.mark.skipif(not os.path.exists(PATH), reason="fixture absent")
@pytest.mark.parametrize("q", ["sg_", "ss_"])
def test_realrun_running_sums_oracle_match_reference(q):
    """The refinement's sumgr and sumsq (epsr_standalone_rev3.py:3578 / :3642) on the loop's
    running means and error bars (accumulated over the run folder's earlier iterations) with the
    real*8 weights fc1, fc2: every updated point, bit for bit."""
    z = np.load(PATH)
    n = int(z[q + "n"])
    fc1, fc2 = (float(v) for v in z[q + "fc"])
    if q == "sg_":
        names = ("gorintra", "gorinter", "gr2intra", "gr2inter", "entsig")
        got = oracle.sumgr(n, z[q + "sample"], z[q + "ycoh"], fc1, fc2, {k: z[q + k + "_in"] for k in names})
    else:
        names = ("soqintra", "soqinter", "sq2intra", "sq2inter")
        got = oracle.sumsq(n, z[q + "sample"], fc1, fc2, {k: z[q + k + "_in"] for k in names})
    for k in names:
        assert_bits_equal(got[k][:, 1:], z[q + k][:, 1:], q + k)
    assert any(not np.array_equal(z[q + k + "_in"], z[q + k]) for k in names)


@pytest.mark.skipif(not os.path.exists(PATH), reason="fixture absent")
def test_realrun_gensq_oracle_matches_reference():
    """The refinement's gensq (epsr_standalone_rev3.py:4731) on the histograms atogen had just
    made, at every 20th Q point of the run's grid (each point reads only its own column of the
    sine-transform table): intra- and intermolecular S(Q), bit for bit."""
    z = np.load(PATH)
    cols = z["gs_foqols"]
    rows = np.zeros((cols.shape[0] + 1, cols.shape[1]), f32)
    rows[1:] = cols
    got = oracle.gensq(cols.shape[0], int(z["gs_npt1"]), z["gs_wav"], rows, z["gs_ycoh"], z["gs_n2extr"],
                       z["gs_natomsphere"])
    assert_bits_equal(got[:, :, 1:], z["gs_sofq"], "sofq")
    assert float(np.abs(z["gs_sofq"][1]).max()) > 0


STOG_PATH = os.path.join(GOLDEN, "realrun_stog.npz")


@pytest.mark.skipif(not os.path.exists(STOG_PATH), reason="fixture absent")
def test_realrun_stog_oracle_matches_reference():
    """The final output section's first stog (ato_manipulation_rev4.py:4067, from
    epsr_standalone_rev3.py:2195) on the fits to the run's three data sets, captured by
    tests/golden/make_golden_realrun_files.py: g(r) of every set at every r point."""
    z = np.load(STOG_PATH)
    got = oracle.stog(f32(z["st_rho"]), z["st_q"], z["st_sofq"], z["st_r"], z["st_nqmin"], z["st_nqmax"], z["st_xwt"])
    assert_bits_equal(got[:, 1:], z["st_gofr"], "gofr")
    assert float(np.abs(z["st_gofr"]).max()) > 0


@pytest.mark.skipif(not os.path.exists(PATH), reason="fixture absent")
def test_realrun_cell_list_oracle_matches_reference():
    """The loop's first initialise_cellneighbourlist (cellneighbourlist.py:23, from
    epsr_standalone_rev3.py:1265) with its nmolcellin and sepmax: divisions, cell count,
    neighbour offsets, the molecules of every cell in the reference's order and each
    molecule's cell."""
    z = np.load(PATH)
    box = _box(z, "cl0_")
    c = oracle.cell_list(box, int(z["cl0_nmolcellin"]), f32(z["cl0_rmax"]))
    dims = [c["ncelldiva"], c["ncelldivb"], c["ncelldivc"], c["ncell"], c["ncellneighb"], c["maxcellno"]]
    assert np.array_equal(np.array(dims, np.int32), z["cl0_dims"])
    nc, nb = int(c["ncell"]), int(c["ncellneighb"])
    assert np.array_equal(c["cell_start"][: nc + 1], z["cl0_cell_start"])
    assert np.array_equal(c["cell_mols"], z["cl0_cell_mols"])
    assert np.array_equal(c["molcellno"], z["cl0_molcellno"])
    off = np.stack([c[k][:nb] for k in ("ia_off", "ib_off", "ic_off")], 1)
    assert np.array_equal(off, z["cl0_offsets"])
    assert nc > 1
