"""Device path vs the reference's golden vectors and the C oracle (needs a B200).

Bit-identical where the reference's arithmetic has no transcendental (ran1, cell list,
pair store, energies, histograms, gensq); the Monte Carlo chain is bit-identical when the
reference's own cosines are injected, and otherwise checked against an FP64 restatement
with the north-star tolerance (1e-5 relative to the energy scale of the move).
"""

import numpy as np
import pytest
import torch

from epsr_python_translation_b200.box import BoxArrays, Ran1State, trsteps
from oracle import oracle
from tests import goldens
from tests.goldens import assert_bits_equal
from tests.chain_check import check_decisions

pytestmark = pytest.mark.gpu
f32 = np.float32

ENERGY_RTOL = 1e-5   # relative to the sum of |pair energies| of the move


def _device(box):
    from epsr_python_translation_b200.device import DeviceBox
    return DeviceBox(box)


def _prepare(case, strict=True):
    z = goldens.load(case)
    box = BoxArrays.from_golden(z)
    d = _device(box)
    d.cell_list(int(z["in_nmolcell"]), f32(z["in_sepmax"]))
    d.fmolec1(z["in_eintra"], strict=strict)
    return z, box, d


# ----------------------------------------------------------------------------- ran1
def test_ran1_device_matches_gfortran_blocks():
    from epsr_python_translation_b200.device import DeviceBox  # noqa: F401  (loads the library)
    from epsr_python_translation_b200 import _lib
    _lib.load(require_device=True)
    z = np.load(goldens.GOLDEN + "/ran1_reference.npz")
    st = None
    for k in range(int(z["nblocks"])):
        head = str(z[f"block{k}_header"])
        if head.startswith("seed"):
            st = torch.from_numpy(Ran1State(idum=int(head.split()[1])).as_array()).cuda()
        out = torch.empty(1000, dtype=torch.float32, device="cuda")
        import ctypes as C
        _lib.check(_lib.load().epsr_ran1_fill(C.c_void_p(st.data_ptr()), C.c_void_p(out.data_ptr()), 1000, None))
        torch.cuda.synchronize()
        assert np.array_equal(out.cpu().numpy().view(np.uint32), z[f"block{k}_bits"]), head
        s = st.cpu().numpy()
        state = z[f"block{k}_state"]
        assert [int(s[2]), int(s[0]), int(s[1])] == [int(v) for v in state[:3]], head
        assert np.array_equal(s[3:35], state[3:35].astype(np.int32)), head


@pytest.mark.parametrize("n", [1, 31, 32, 33, 1000, 100003])
def test_ran1_device_lengths_match_oracle(n):
    from epsr_python_translation_b200.device import DeviceBox
    z = goldens.load("c1_water")
    d = DeviceBox(BoxArrays.from_golden(z))
    st0 = Ran1State.from_golden(z, "mf_ran1_before_")
    t = d.ran1_tensor(st0)
    vals = d.ran1_fill(t, n)
    ref, rst = oracle.ran1_fill(st0, n)
    assert np.array_equal(vals.cpu().numpy().view(np.uint32), ref.view(np.uint32))
    assert np.array_equal(t.cpu().numpy(), rst.as_array())


# ----------------------------------------------------------------------------- cells + store
@pytest.mark.parametrize("case", goldens.CASES)
def test_cell_list_device_matches_reference(case):
    z = goldens.load(case)
    d = _device(BoxArrays.from_golden(z))
    d.cell_list(int(z["in_nmolcell"]), f32(z["in_sepmax"]))
    c = d.download_cells()
    for k in ("ncelldiva", "ncelldivb", "ncelldivc", "ncell", "maxcellno", "ncellneighb"):
        assert c[k] == int(z["cell_" + k]), k
    start, flat = goldens.golden_cells_csr(z)
    assert np.array_equal(c["cell_start"], start)
    assert np.array_equal(c["cell_mols"], flat)
    assert np.array_equal(c["molcellno"], z["cell_molcellno"])
    assert np.array_equal(c["offsets"][:, 0], z["cell_iacellneighb"])
    assert np.array_equal(c["offsets"][:, 1], z["cell_ibcellneighb"])
    assert np.array_equal(c["offsets"][:, 2], z["cell_iccellneighb"])
    assert c["nnbrefmax"] == int(z["fm_nnbrefmax"])


@pytest.mark.parametrize("case", goldens.CASES)
def test_fmolec1_device_store_matches_reference(case):
    z, box, d = _prepare(case)
    st = d.download_store()
    assert st["nergpair"] == int(z["fm_nergpair"])
    assert np.array_equal(st["nergpairm"], z["fm_nergpairm"])
    for im in range(box.nmol):
        k = st["nergpairm"][im]
        assert np.array_equal(st["molergpair"][im, :k], z["fm_molergpair"][:k, im] - 1), im
        assert np.array_equal(st["ergpairref"][im, :k], z["fm_ergpairref"][:k, im]), im
    assert_bits_equal(st["ergpair"], z["fm_ergpair"], "ergpair")


def test_fmolec1_device_sums_strict_and_fast():
    z = goldens.load("c2_mixture")
    box = BoxArrays.from_golden(z)
    d = _device(box)
    d.cell_list(int(z["in_nmolcell"]), f32(z["in_sepmax"]))
    ft, fb = d.fmolec1(z["in_eintra"], strict=True)
    assert_bits_equal(ft, z["fm_ftest"], "ftest")
    assert_bits_equal(fb, z["fm_ftestb"], "ftestb")
    ft2, fb2 = d.fmolec1(z["in_eintra"], strict=False)
    # fast mode sums in double: compare with the exact sum of the stored float32 energies
    st = d.download_store()
    nintra = int(np.count_nonzero(z["in_eintra"]))
    exact = float(np.sum(st["ergpair"][nintra:].astype(np.float64))) / box.nmol
    scale = float(np.sum(np.abs(st["ergpair"][nintra:].astype(np.float64)))) / box.nmol
    assert abs(float(ft2) - exact) <= 1e-6 * scale + 1e-6
    exactb = float(np.sum(z["in_eintra"].astype(np.float64))) / box.nmol
    assert abs(float(fb2) - exactb) <= 1e-6 * abs(exactb) + 1e-12


# ----------------------------------------------------------------------------- molfit
def _mc(d, z, box):
    tmax, tmin = trsteps(box.natomr)
    nmt = box.nmoltype
    d.mc_setup(rejrate=f32(z["in_rejrate"]), stepr=f32(z["in_stepr"]), stepm=f32(z["in_stepm"]),
               wholerot=z["in_wholerot"], wholetrans=z["in_wholetrans"], internrot=np.zeros(nmt, f32),
               interntrans=np.zeros(nmt, f32), ran1=Ran1State.from_golden(z, "mf_ran1_before_"), trstepmax=tmax,
               trstepmin=tmin)


@pytest.mark.parametrize("case", goldens.CASES)
def test_molfit_device_bit_identical_with_reference_cosines(case):
    """With the reference's own cosf values injected, every coordinate, stored energy, step
    size, counter and the ran1 state match the reference bit for bit."""
    z, box, d = _prepare(case)
    _mc(d, z, box)
    for cyc in range(int(z["mf_cycles"])):
        p = f"mf{cyc}_"
        d.molfit(strict=True, cos_override=z[p + "cos"])
        m = d.download_mc()
        assert_bits_equal(m["den"], z[p + "den"], p + "den")
        co = d.download_coords()
        for k in ("xa", "ya", "za", "xadd", "yadd", "zadd"):
            assert_bits_equal(co[k], z[p + k], p + k)
        st = d.download_store()
        assert_bits_equal(st["ergpair"], z[p + "ergpair"], p + "ergpair")
        assert_bits_equal(m["wholerot"], z[p + "wholerot"], p + "wholerot")
        assert_bits_equal(m["wholetrans"], z[p + "wholetrans"], p + "wholetrans")
        assert np.array_equal(m["nwhole"], z[p + "nwhole"])
        assert np.array_equal(m["nmovem"], z[p + "nmovem"])
        assert np.array_equal(m["nstepreject"], z[p + "nstepreject"])
        assert_bits_equal(m["fadds"], z[p + "fadds"], p + "fadds")
        assert m["ran1"].idum == int(z[p + "ran1_after_idum"])
        assert np.array_equal(m["ran1"].iv, z[p + "ran1_after_iv"])


@pytest.mark.parametrize("case", goldens.CASES)
def test_molfit_fast_path_matches_reference_with_reference_cosines(case):
    """The speculative cycle (all proposals and pair energies in parallel, decisions resolved
    in visit order, each move's change summed in double): coordinates, stored energies, step
    sizes, counters and the ran1 state equal the reference's; the per-move change is within
    the energy tolerance of the reference's float32 sum."""
    z, box, d = _prepare(case)
    _mc(d, z, box)
    ob = BoxArrays.from_golden(z)
    oc = oracle.cell_list(ob, int(z["in_nmolcell"]), f32(z["in_sepmax"]))
    ost = oracle.fmolec1(ob, oc, z["in_eintra"])
    nmt = box.nmoltype
    omc = dict(rejrate=f32(z["in_rejrate"]), stepr=f32(z["in_stepr"]), stepm=f32(z["in_stepm"]),
               wholerot=z["in_wholerot"].copy(), wholetrans=z["in_wholetrans"].copy(),
               internrot=np.zeros(nmt, f32), interntrans=np.zeros(nmt, f32), ireset=0)
    ran1 = Ran1State.from_golden(z, "mf_ran1_before_")
    for cyc in range(int(z["mf_cycles"])):
        p = f"mf{cyc}_"
        d.molfit(strict=False, cos_override=z[p + "cos"])
        d.check_status()
        m = d.download_mc()
        _, tr, ran1 = oracle.molfit(ob, oc, ost, omc, ran1)
        tol = ENERGY_RTOL * tr["scale64"] + 1e-6
        assert np.all(np.abs(m["den"].astype(np.float64) - tr["den64"]) <= tol), cyc
        assert np.array_equal(m["acc"], z[p + "den"].shape[0] and tr["acc"]), cyc
        co = d.download_coords()
        for k in ("xa", "ya", "za", "xadd", "yadd", "zadd"):
            assert_bits_equal(co[k], z[p + k], p + k)
        st = d.download_store()
        assert_bits_equal(st["ergpair"], z[p + "ergpair"], p + "ergpair")
        assert_bits_equal(m["wholerot"], z[p + "wholerot"], p + "wholerot")
        assert_bits_equal(m["wholetrans"], z[p + "wholetrans"], p + "wholetrans")
        assert np.array_equal(m["nwhole"], z[p + "nwhole"])
        assert np.array_equal(m["nmovem"], z[p + "nmovem"])
        assert np.array_equal(m["nstepreject"], z[p + "nstepreject"])
        assert abs(float(m["fadds"]) - float(z[p + "fadds"])) <= 1e-5 * max(1.0, abs(float(z[p + "fadds"])))
        assert m["ran1"].idum == int(z[p + "ran1_after_idum"])
        assert np.array_equal(m["ran1"].iv, z[p + "ran1_after_iv"])


def _check_chain(case, strict):
    """Device cosines: energies within ENERGY_RTOL of the FP64 restatement; every decision is
    the Metropolis rule applied to the device's own energy change and the draw of the shared
    ran1 stream; and a decision differs from the reference's only where the Metropolis
    threshold -simt*ln(u) of that draw lies within the energy tolerance of the exact change
    (the chains then part, and the comparison stops)."""
    z, box, d = _prepare(case)
    _mc(d, z, box)
    ob = BoxArrays.from_golden(z)
    oc = oracle.cell_list(ob, int(z["in_nmolcell"]), f32(z["in_sepmax"]))
    ost = oracle.fmolec1(ob, oc, z["in_eintra"])
    nmt = box.nmoltype
    omc = dict(rejrate=f32(z["in_rejrate"]), stepr=f32(z["in_stepr"]), stepm=f32(z["in_stepm"]),
               wholerot=z["in_wholerot"].copy(), wholetrans=z["in_wholetrans"].copy(),
               internrot=np.zeros(nmt, f32), interntrans=np.zeros(nmt, f32), ireset=0)
    ran1 = Ran1State.from_golden(z, "mf_ran1_before_")
    for cyc in range(int(z["mf_cycles"])):
        d.molfit(strict=strict)
        m = d.download_mc()
        _, tr, ran1 = oracle.molfit(ob, oc, ost, omc, ran1)
        if check_decisions(m["den"], m["acc"], tr, box.simt, ENERGY_RTOL) == "parted":
            return
        co = d.download_coords()
        for kk in ("xadd", "yadd", "zadd", "xa", "ya", "za"):
            assert np.max(np.abs(co[kk] - getattr(ob, kk))) < 1e-5, kk


@pytest.mark.parametrize("case", goldens.CASES)
def test_molfit_device_cos_strict_chain(case):
    _check_chain(case, strict=True)


@pytest.mark.parametrize("case", goldens.CASES)
def test_molfit_device_fast_sum_chain(case):
    _check_chain(case, strict=False)


def test_en_change_and_en_mole_pair_entry_points():
    z, box, d = _prepare("mix_small")
    import ctypes as C
    from epsr_python_translation_b200 import _lib
    lib = _lib.load()
    M = d.nnbrefmax
    erg = torch.zeros(M, dtype=torch.float32, device="cuda")
    out = np.zeros(1, f32)
    ob = BoxArrays.from_golden(z)
    oc = oracle.cell_list(ob, int(z["in_nmolcell"]), f32(z["in_sepmax"]))
    ost = oracle.fmolec1(ob, oc, z["in_eintra"])
    for im in (0, 7, box.nmol - 1):
        _lib.check(lib.epsr_en_change(C.byref(d.cbox), C.byref(d.store), im, C.c_void_p(erg.data_ptr()),
                                      out.ctypes.data_as(C.c_void_p), None))
        ref, _, _, ref_new = oracle.en_change(ob, ost, im)
        assert_bits_equal(out[0], ref, f"en_change {im}")
        n = int(ost["nergpairm"][im])
        assert_bits_equal(erg.cpu().numpy()[1:n], ref_new[1:n], f"ergnew {im}")
    ims = torch.tensor([0, 1, 2, 10], dtype=torch.int32, device="cuda")
    jms = torch.tensor([5, 9, 33, 40], dtype=torch.int32, device="cuda")
    res = torch.zeros(4, dtype=torch.float32, device="cuda")
    _lib.check(lib.epsr_en_mole_pair(C.byref(d.cbox), C.c_void_p(ims.data_ptr()), C.c_void_p(jms.data_ptr()), 4,
                                     C.c_void_p(res.data_ptr()), None))
    r = res.cpu().numpy()
    for k, (i, j) in enumerate(zip([0, 1, 2, 10], [5, 9, 33, 40])):
        assert_bits_equal(r[k], oracle.en_mole_pair(ob, i, j), f"pair {i},{j}")


# ----------------------------------------------------------------------------- atogen
@pytest.mark.parametrize("case", goldens.CASES)
def test_atogen_device_matches_reference(case):
    z = goldens.load(case)
    box = BoxArrays.from_golden(z)
    last = int(z["mf_cycles"]) - 1
    for k in ("xa", "ya", "za", "xadd", "yadd", "zadd"):
        setattr(box, k, z[f"mf{last}_{k}"].copy())
    d = _device(box)
    t = d.ran1_tensor(Ran1State.from_golden(z, "ag_ran1_before_"))
    ngr = d.atogen(int(z["ag_ngrsamples_in"]), t, z["ag_rminex"])
    assert ngr == int(z["ag_ngrsamples"])
    wav, potex = d.download_wav()
    mine = wav[:, :, 1:box.npt1 + 1].transpose(0, 2, 1)
    assert_bits_equal(mine, z["ag_wav"], "wav")
    assert_bits_equal(potex, z["ag_potex"], "potex")
    s = t.cpu().numpy()
    assert int(s[0]) == int(z["ag_ran1_after_idum"]) and np.array_equal(s[3:35], z["ag_ran1_after_iv"])
    assert d.last_pair_updates > 0


# ----------------------------------------------------------------------------- gensq / stog
@pytest.mark.parametrize("case", ["c1_water", "mix_small"])
def test_gensq_device_matches_reference(case):
    from epsr_python_translation_b200 import transforms
    z = goldens.load(case)
    box = BoxArrays.from_golden(z)
    npt1, nq = box.npt1, int(z["gs_nq"])
    ld = box.npt + 1
    wav = np.zeros((2, box.npairs, ld), f32)
    wav[:, :, 1:npt1 + 1] = z["ag_wav"].transpose(0, 2, 1)
    F = np.ascontiguousarray(z["gs_foqols"])   # (npt1+1, nq+1): F[j, i], i fastest
    out = transforms.gensq(nq, npt1, torch.from_numpy(wav.reshape(-1)).cuda(), ld, F, nq + 1, 1,
                           z["gs_ycoh"][:ld] if z["gs_ycoh"].shape[0] >= ld else np.pad(z["gs_ycoh"], (0, ld)),
                           box.n2extr, np.ones(box.ntype, f32), box.npairs)
    o = out.cpu().numpy().reshape(2, box.npairs, nq + 1)
    assert_bits_equal(o[:, :, 1:].transpose(0, 2, 1), z["gs_sofq"], "sofq")


@pytest.mark.parametrize("case", ["c1_water", "mix_small"])
def test_stog_device_within_tolerance(case):
    """The sine is the only transcendental; each g(r) value is checked against the
    reference within 1e-5 of the magnitude of its summed terms."""
    from epsr_python_translation_b200 import transforms
    z = goldens.load(case)
    q = z["gs_q"]
    nq = q.shape[0] - 1
    sofq = z["gs_sofq"][1]
    sp = np.zeros((sofq.shape[1], nq + 1), f32)
    sp[:, 1:] = sofq.T
    r = np.zeros(z["sg_r"].shape[0] + 1, f32)
    r[1:] = z["sg_r"]
    g = transforms.stog(f32(z["sg_rho"]), q, sp, r, z["sg_nqmin"], z["sg_nqmax"], z["sg_xwt"]).cpu().numpy()
    ref = z["sg_gofr"]
    qq = q.astype(np.float64)
    rho = float(z["sg_rho"])
    sfac = 0.5 * (qq[4] - qq[3]) / np.pi / np.pi / rho
    for j in range(1, r.shape[0]):
        rr = max(float(r[j]), 1e-30)
        scale = sfac * np.sum(np.abs(sp[:, 2:] * qq[2:] * (qq[2:] if r[j] == 0 else 1.0)), axis=1) / (
            rr if r[j] > 0 else 1.0)
        tol = 1e-5 * (scale + np.abs(z["sg_xwt"])) + 1e-7
        diff = np.abs(g[:, j] - ref[j - 1])
        assert np.all(diff <= tol), (j, diff.max(), tol.min())


# ----------------------------------------------------------------------------- fit_expansion
@pytest.mark.parametrize("run", [0, 1])
def test_fit_expansion_device_matches_reference(run):
    from epsr_python_translation_b200 import transforms
    from epsr_python_translation_b200.device import DeviceBox  # noqa: F401
    z = np.load(goldens.GOLDEN + "/fitexp.npz")
    p = f"fx{run}_"
    nterms, npt = int(z["fx_nterms"]), int(z["fx_npt"])
    wtold = np.zeros(nterms + 1, f32)
    wtold[1:] = z[p + "wtold_in"]
    st = torch.from_numpy(Ran1State.from_golden(z, p + "ran1_before_").as_array()).cuda()
    res = transforms.fit_expansion(z["fx_yin"], z["fx_expr"], wtold, f32(z["fx_stepr_in"]), 1, npt,
                                   int(z[p + "ncfirst"]), nterms, 1000, int(z["fx_nfreq"]), st)
    assert_bits_equal(res["wt"].cpu().numpy()[1:], z[p + "wt"], "wt")
    assert_bits_equal(res["wtold"].cpu().numpy()[1:], z[p + "wtold"], "wtold")
    assert_bits_equal(res["yout"].cpu().numpy()[1:], z[p + "yout"], "yout")
    for k in ("stepr", "acceptr", "rejrat", "chisq"):
        assert_bits_equal(res[k], z[p + k], k)
    s = st.cpu().numpy()
    assert int(s[0]) == int(z[p + "ran1_after_idum"]) and int(s[2]) == int(z[p + "ran1_after_mcall"])


@pytest.mark.parametrize("strict", [True, False])
def test_fit_expansion_batch_equals_successive_calls(strict):
    """One launch over three data sets equals three successive calls on the same ran1
    stream (the reference's ptgnsq loop), bit for bit, in both summation modes; the C2-size
    basis (600 Q rows x 116 terms) runs on a two-CTA cluster."""
    from epsr_python_translation_b200 import configs, transforms
    wl = configs.make_workload("c2_mixture")
    nq, nt = wl.nq, wl.nterms
    rng = np.random.default_rng(3)
    ndata = 3
    yin = np.zeros((ndata, nq + 1), f32)
    yin[:, 1:] = (rng.standard_normal((ndata, nq)) * 0.05).astype(f32)
    wtold = np.zeros((ndata, nt + 1), f32)
    wtold[:, 1:] = (rng.standard_normal((ndata, nt)) * 0.01).astype(f32)
    stepr = np.array([0.01, 0.02, 0.005], f32)
    seed = Ran1State(idum=-99)
    st1 = torch.from_numpy(seed.as_array()).cuda()
    single = []
    for k in range(ndata):
        single.append(transforms.fit_expansion(yin[k], wl.expr, wtold[k], stepr[k], 1, nq, 1, nt, 1000, 10, st1,
                                               strict=strict))
    st2 = torch.from_numpy(seed.as_array()).cuda()
    b = transforms.fit_expansion_batch(yin, wl.expr, wtold, stepr, 1, nq, 1, nt, 1000, 10, st2, strict=strict)
    for k in range(ndata):
        for name in ("wt", "wtold", "yout"):
            assert_bits_equal(b[name][k].cpu().numpy(), single[k][name].cpu().numpy(), f"{name} {k}")
        for name in ("stepr", "acceptr", "rejrat", "chisq"):
            assert_bits_equal(b[name][k], single[k][name], f"{name} {k}")
        assert int(b["trials"][k]) == single[k]["trials"]
    assert np.array_equal(st1.cpu().numpy(), st2.cpu().numpy())


@pytest.mark.parametrize("seed", [3, 4])
def test_fit_expansion_c2_size_strict_matches_oracle(seed):
    """At the C2 size (600 Q rows x 116 terms, 116 draws per trial, a two-CTA cluster whose
    CTAs each generate the ran1 stream in a warp of their own) the strict fit equals the C
    oracle bit for bit: coefficients, fitted curve, step, rates, chi^2 and the ran1 state."""
    from epsr_python_translation_b200 import configs, transforms
    wl = configs.make_workload("c2_mixture")
    nq, nt = wl.nq, wl.nterms
    rng = np.random.default_rng(seed)
    yin = np.zeros(nq + 1, f32)
    yin[1:] = (rng.standard_normal(nq) * 0.05).astype(f32)
    wtold = np.zeros(nt + 1, f32)
    wtold[1:] = (rng.standard_normal(nt) * 0.01).astype(f32)
    st0 = Ran1State(idum=-seed)
    t = torch.from_numpy(st0.as_array()).cuda()
    res = transforms.fit_expansion(yin, wl.expr, wtold, f32(0.01), 1, nq, 1, nt, 1000, 10, t, strict=True)
    ref, rst = oracle.fit_expansion(yin, wl.expr, wtold.copy(), f32(0.01), 1, nq, 1, nt, 1000, 10, st0)
    assert_bits_equal(res["wt"].cpu().numpy()[1:], ref["wt"][1:], "wt")
    assert_bits_equal(res["wtold"].cpu().numpy()[1:], ref["wtold"][1:], "wtold")
    assert_bits_equal(res["yout"].cpu().numpy()[1:], ref["yout"][1:], "yout")
    for k in ("stepr", "acceptr", "rejrat", "chisq"):
        assert_bits_equal(res[k], ref[k], k)
    assert res["trials"] == ref["trials"]
    assert np.array_equal(t.cpu().numpy(), rst.as_array())


@pytest.mark.parametrize("seed,npt", [(3, 600), (4, 600), (5, 600), (6, 1000)])
def test_fit_expansion_fast_mode_matches_oracle(seed, npt):
    """The fast fit (the mode the iteration and the benchmark run: chi^2 of each trial summed
    in double over the rows and rounded once to float32) against the C oracle's restatement
    of that summation, bit for bit: coefficients, fitted curve, step, rates, final chi^2,
    trial count and the ran1 state.  The oracle's own fast chains are checked against its
    reference-order chains in tests/test_fit_fast_statistics.py."""
    from epsr_python_translation_b200 import configs, transforms
    nt = 116
    q = configs.qgrid(npt, 0.05)
    expr = configs.ep_basis(q, nt)
    rng = np.random.default_rng(seed)
    yin = np.zeros(npt + 1, f32)
    yin[1:] = (rng.standard_normal(npt) * 0.05).astype(f32)
    wtold = np.zeros(nt + 1, f32)
    wtold[1:] = (rng.standard_normal(nt) * 0.01).astype(f32)
    st0 = Ran1State(idum=-seed)
    t = torch.from_numpy(st0.as_array()).cuda()
    res = transforms.fit_expansion(yin, expr, wtold, f32(0.01), 1, npt, 1, nt, 1000, 10, t, strict=False)
    ref, rst = oracle.fit_expansion(yin, expr, wtold.copy(), f32(0.01), 1, npt, 1, nt, 1000, 10, st0, fast=True)
    assert_bits_equal(res["wt"].cpu().numpy()[1:], ref["wt"][1:], "wt")
    assert_bits_equal(res["wtold"].cpu().numpy()[1:], ref["wtold"][1:], "wtold")
    assert_bits_equal(res["yout"].cpu().numpy()[1:], ref["yout"][1:], "yout")
    for k in ("stepr", "acceptr", "rejrat", "chisq"):
        assert_bits_equal(res[k], ref[k], k)
    assert res["trials"] == ref["trials"]
    assert np.array_equal(t.cpu().numpy(), rst.as_array())


@pytest.mark.parametrize("npt,scale", [(1000, 1.0), (1700, 1.0), (600, 3.0e12)])
def test_fit_expansion_cluster_shapes_strict_match_oracle(npt, scale):
    """Cluster shapes of the fit against the C oracle, strict sums, bit for bit: 1000 Q rows
    (the C3 S(Q)) on three CTAs, 1700 rows on four (odd row counts per CTA, so the exchange
    buffers need their padding), and a basis scaled so that row sums reach the clamp level
    (e^25), which takes the clamped sum for those rows."""
    from epsr_python_translation_b200 import configs, transforms
    nt = 116
    q = configs.qgrid(npt, 0.05)
    expr = configs.ep_basis(q, nt)
    if scale != 1.0:
        expr = (expr * f32(scale)).astype(f32)
    rng = np.random.default_rng(npt)
    yin = np.zeros(npt + 1, f32)
    yin[1:] = (rng.standard_normal(npt) * 0.05 * scale).astype(f32)
    wtold = np.zeros(nt + 1, f32)
    wtold[1:] = (rng.standard_normal(nt) * 0.01).astype(f32)
    st0 = Ran1State(idum=-5)
    t = torch.from_numpy(st0.as_array()).cuda()
    res = transforms.fit_expansion(yin, expr, wtold, f32(0.01), 1, npt, 1, nt, 1000, 10, t, strict=True)
    ref, rst = oracle.fit_expansion(yin, expr, wtold.copy(), f32(0.01), 1, npt, 1, nt, 1000, 10, st0)
    if scale != 1.0:
        assert np.any(np.abs(ref["yout"][1:]) >= np.float32(np.exp(25.0)) * 0.999)   # the clamp acted
    assert_bits_equal(res["wt"].cpu().numpy()[1:], ref["wt"][1:], "wt")
    assert_bits_equal(res["wtold"].cpu().numpy()[1:], ref["wtold"][1:], "wtold")
    assert_bits_equal(res["yout"].cpu().numpy()[1:], ref["yout"][1:], "yout")
    for k in ("stepr", "acceptr", "rejrat", "chisq"):
        assert_bits_equal(res[k], ref[k], k)
    assert res["trials"] == ref["trials"]
    assert np.array_equal(t.cpu().numpy(), rst.as_array())


@pytest.mark.gpu
def test_ptgnsq_difference_bit_identical():
    """The per-data-set simulated fit and its difference from the data (ptgnsq
    epsr_standalone_rev3.py:3844-3867) equals the oracle's sequential sum (real*8 weights, one
    float32 rounding per pair) bit for bit; the weights are general doubles."""
    from epsr_python_translation_b200 import transforms
    rng = np.random.default_rng(11)
    ndata, npairs, nq = 3, 21, 600
    data = rng.standard_normal((ndata, nq + 1)).astype(f32)
    cwt = rng.uniform(0.0, 0.2, (ndata, npairs))
    qwind = (rng.standard_normal((npairs, nq + 1)) * 0.3).astype(f32)
    got = transforms.ptgnsq_difference(torch.from_numpy(data).cuda(), torch.from_numpy(cwt).cuda(),
                                       torch.from_numpy(qwind).cuda()).cpu().numpy()
    assert_bits_equal(got, oracle.ptgnsq_difference(data, cwt, qwind), "ptgnsq difference")


def test_triclinic_minimage_device_matches_reference():
    """The device minimum image on non-cubic lattices (minimagec.py:13-45) against the
    reference's own results (tests/golden/triclinic.npz), bit for bit: every centre of a box
    of single-atom molecules put back in the cell by epsr_minimage_centres."""
    import os
    z = np.load(os.path.join(goldens.GOLDEN, "triclinic.npz"))
    for case in z["cases"]:
        box = goldens.point_box(z[f"{case}_lat6"], z[f"{case}_pts"])
        d = _device(box)
        d.minimage_centres()
        co = d.download_coords()
        got = np.stack([co["xadd"], co["yadd"], co["zadd"]], axis=1)
        assert_bits_equal(got, z[f"{case}_out"], str(case))
