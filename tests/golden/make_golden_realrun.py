"""Golden vectors taken from inside the reference's own epsr loop on its shipped run folder
(EPSR-test: 200 DMSO + 400 water with the DMSO methyl groups as ROT groups), made by running
the reference translation (epsr26) itself.

    EPSR_REFERENCE=<reference checkout> PYTHONDONTWRITEBYTECODE=1 python tests/golden/make_golden_realrun.py

The run folder is copied to a scratch directory, its input file's niter raised to 2
(prepare_run), and the unchanged epsr program runs on it (runepsr17
epsr_standalone_rev3.py:1235: the files read, the potentials built, the cell list, fmolec1,
molfit ntimes times, the refinement, again).  Three molfit calls are captured through the
module attribute the loop calls (molfit.molfit, as the reference's tracer reroutes routines):
the run folder's nisum starts at intra, so the first is the intramolecular cycle, each
molecule's atoms moved and then its methyl groups rotated (molfit.py:124-267); the second a
whole-molecule cycle (:268-448); the sixth, after the first refinement, a whole-molecule cycle
with the internal rotations of the methyl groups (:295-360).  For each, everything that call
reads is written before it and everything it changes after it (every array copied, the
COMMON arrays being updated in place): the box as the COMMON blocks hold it (read by the
drop-in's own box_from_common), the cell list as the loop built it, the pair store, the step
arrays and counters, the rotational groups and the intramolecular model, the ran1 state, the
call's arguments and results, and the cosines molfit drew.  The loop's first cell list
(prefix cl0_) and the refinement's first atogen,
press and fit_expansion calls, its running sums and its generate_ep call are captured the
same way, and its gensq at every 20th Q point.  The run is stopped after the sixth molfit call.
tests/golden/realrun.npz receives the molfit calls under the prefixes k0_, k1_, k2_ and the
atogen, press, gensq, fit_expansion, sumsq, sumgr and generate_ep calls under ag_, pr_, gs_,
fx_, ss_, sg_ and ge_.
"""

from __future__ import annotations

import os
import shutil
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)
sys.path.insert(0, HERE)

import refstate  # noqa: E402

f32 = np.float32
REF = refstate.reference_root()


class _Stop(Exception):
    pass


# the molfit calls captured (1-based, in the loop's order): the first intramolecular cycle, the
# whole-molecule cycle after it, and the first whole-molecule cycle with internal rotations
# (nisum 5 = rotfreq), which comes after the first potential refinement
CAPTURE = (1, 2, 6)
NITER = 2


def prepare_run(run):
    """The run folder as the captures need it: the input file's niter raised to NITER, so
    that the loop refines the potential once and reaches the sixth molfit call."""
    import re
    inp = os.path.join(run, "200DMSO400Water.EPSR.inp")
    with open(inp) as f:
        text = f.read()
    text, n = re.subn(r"^(niter\s+)\d+", lambda m: m.group(1) + str(NITER), text, count=1, flags=re.M)
    if n != 1:
        raise SystemExit("no niter line in " + inp)
    with open(inp, "w") as f:
        f.write(text)


def _fortran_slice(a, *dims):
    """The 1-based part of a reference array, 0-based, as a copy."""
    return np.array(np.asarray(a)[tuple(slice(1, d + 1) for d in dims)])


def snapshot(common, mods, out, q):
    """Everything one molfit call reads from the COMMON blocks, under prefix q."""
    from epsr_python_translation_b200 import dropin
    p = dropin.PairPath(common, mods)
    box = p.box_from_common()
    for k, v in box.__dict__.items():
        if isinstance(v, np.ndarray):
            out[q + "box_" + k] = v.copy()
        else:
            out[q + "box_" + k] = np.array(v)
    cc, mc, e16, erd, cnl = common.clustercom, common.molecom, common.epsr16, common.ergpairreference, \
        common.cellneighbourlist
    nmol, nmt = int(cc.nmol), int(cc.nmoltype)
    # the pair store
    M = int(erd.nnbrefmax)
    out[q + "st_nnbrefmax"], out[q + "st_nergpair"] = np.int32(M), np.int32(erd.nergpair)
    out[q + "st_nergpairm"] = np.array(erd.nergpairm[1:nmol + 1], np.int32)
    out[q + "st_molergpair"] = _fortran_slice(erd.molergpair, M, nmol).T.astype(np.int32) - 1
    out[q + "st_ergpairref"] = _fortran_slice(erd.ergpairref, M, nmol).T.astype(np.int32)
    out[q + "st_ergpair"] = np.array(erd.ergpair[1:int(erd.nergpair) + 1], f32)
    # the cell list as the loop built it (cells in reference order, 1-based molecules)
    ncell = int(cnl.ncell)
    n_in = np.array(cnl.nmolsincell[1:ncell + 1], np.int32)
    mols = [np.array(cnl.molsincell[1:n_in[c] + 1, c + 1], np.int32) - 1 for c in range(ncell)]
    out[q + "cl_dims"] = np.array([cnl.ncelldiva, cnl.ncelldivb, cnl.ncelldivc, ncell, cnl.ncellneighb,
                                   cnl.maxcellno], np.int32)
    out[q + "cl_cell_start"] = np.concatenate([[0], np.cumsum(n_in)]).astype(np.int32)
    out[q + "cl_cell_mols"] = np.concatenate(mols).astype(np.int32) if mols else np.zeros(0, np.int32)
    out[q + "cl_molcellno"] = np.array(cnl.molcellno[1:nmol + 1], np.int32)
    nb = int(cnl.ncellneighb)
    out[q + "cl_offsets"] = np.stack([np.array(getattr(cnl, k)[1:nb + 1], np.int32)
                                      for k in ("iacellneighb", "ibcellneighb", "iccellneighb")], 1)
    # step arrays, counters, parameters
    for k in ("wholerot", "wholetrans", "internrot", "interntrans"):
        out[q + k] = np.array(getattr(cc, k)[1:nmt + 1], f32)
    out[q + "nstepreject"] = np.array(cc.nstepreject[1:nmol + 1], np.int32)
    out[q + "ngrot"] = np.array(cc.ngrot[1:nmol + 1], np.int32)
    out[q + "par"] = np.array([e16.rejrate, mc.stepr, mc.stepm, mc.stepri, mc.stepmi], f32)
    g = p._rot_groups()
    if g:
        for k, v in zip(("rot_nrf", "rot_nrl", "rot_axis", "rot_first", "rot_last", "rot_atoms"), g):
            out[q + k] = np.array(v, np.int32)
    for k, v in refstate.ran1_state().items():
        out[q + "ran1_before_" + k] = v


def box_snapshot(common, mods, out, q):
    """The box as the COMMON blocks hold it and the ran1 state, under prefix q."""
    from epsr_python_translation_b200 import dropin
    for k, v in dropin.PairPath(common, mods).box_from_common().__dict__.items():
        out[q + "box_" + k] = v.copy() if isinstance(v, np.ndarray) else np.array(v)
    for k, v in refstate.ran1_state().items():
        out[q + "ran1_before_" + k] = v


def capture_cells(common, mods, out, orig):
    """The loop's first initialise_cellneighbourlist call (cellneighbourlist.py:23, from
    epsr_standalone_rev3.py:1265) under prefix cl0_: the box, nmolcellin and rmax before; the
    cell list it left in the COMMON block after (as snapshot's cl_ arrays)."""
    def wrapped(nmolcellin, xadd, yadd, zadd, nmol, rmax):
        if "cl0_rmax" in out:
            return orig(nmolcellin, xadd, yadd, zadd, nmol, rmax)
        box_snapshot(common, mods, out, "cl0_")
        out["cl0_nmolcellin"] = np.int32(nmolcellin)
        out["cl0_rmax"] = f32(rmax)
        r = orig(nmolcellin, xadd, yadd, zadd, nmol, rmax)
        cnl = common.cellneighbourlist
        ncell = int(cnl.ncell)
        n_in = np.array(cnl.nmolsincell[1:ncell + 1], np.int32)
        out["cl0_dims"] = np.array([cnl.ncelldiva, cnl.ncelldivb, cnl.ncelldivc, ncell, cnl.ncellneighb,
                                    cnl.maxcellno], np.int32)
        out["cl0_cell_start"] = np.concatenate([[0], np.cumsum(n_in)]).astype(np.int32)
        out["cl0_cell_mols"] = np.concatenate([np.array(cnl.molsincell[1:n_in[c] + 1, c + 1], np.int32) - 1
                                               for c in range(ncell)]).astype(np.int32)
        out["cl0_molcellno"] = np.array(cnl.molcellno[1:int(nmol) + 1], np.int32)
        nb = int(cnl.ncellneighb)
        out["cl0_offsets"] = np.stack([np.array(getattr(cnl, k)[1:nb + 1], np.int32)
                                       for k in ("iacellneighb", "ibcellneighb", "iccellneighb")], 1)
        return r
    return wrapped


def capture_atogen(common, mods, out, orig):
    """The loop's first atogen call (ato_manipulation_rev4.py:3640, from
    epsr_standalone_rev3.py:1397) under prefix ag_: the box, the ran1 state, the per-pair
    close-contact radius rminex (of each pair's set), ycoh, sizefactor and ngrsamples before;
    wav (2, npt1, npairs), potex, the returned count and the ran1 state after."""
    def wrapped(wav, ngrsamples):
        if "ag_ngrsamples" in out:
            return orig(wav, ngrsamples)
        pp, e16, mc = common.potential_par, common.epsr16, common.molecom
        npairs, npt1 = int(mc.npairs), int(e16.npt1)
        box_snapshot(common, mods, out, "ag_")
        out["ag_rminex"] = np.array([pp.rminex[int(pp.irefpcof[p + 1])] for p in range(npairs)], f32)
        out["ag_ycoh"] = np.array(e16.ycoh[: int(e16.npt) + 1], f32)
        out["ag_sizefactor"] = f32(mc.sizefactor)
        out["ag_ngrsamples"] = np.int32(ngrsamples)
        n = orig(wav, ngrsamples)
        out["ag_wav"] = np.array(np.asarray(wav)[1:3, 1:npt1 + 1, 1:npairs + 1], f32)
        out["ag_potex"] = np.array(pp.potex[1:npairs + 1], f32)
        out["ag_result"] = np.int32(n)
        for k, v in refstate.ran1_state().items():
            out["ag_ran1_after_" + k] = v
        return n
    return wrapped


def capture_press(common, mods, out, orig):
    """The loop's first press call (ato_manipulation_rev4.py:3903, from
    epsr_standalone_rev3.py:1655) under prefix pr_: the box, cells and pair store before
    (snapshot), npt1, simt and the volume; the returned energy and pressure after."""
    def wrapped(energy, pressc, energf, pressf, energabs, energthreeb, prthreebout):
        if "pr_result" in out:
            return orig(energy, pressc, energf, pressf, energabs, energthreeb, prthreebout)
        snapshot(common, mods, out, "pr_")
        out["pr_scal"] = np.array([common.epsr16.npt1, common.molecom.simt, common.clustercom.volume], f32)
        r = orig(energy, pressc, energf, pressf, energabs, energthreeb, prthreebout)
        out["pr_result"] = np.array([r[0], r[1]], f32)
        return r
    return wrapped


def capture_fit(common, out, orig):
    """The refinement's first fit_expansion call (epsr_standalone_rev3.py:4806, from ptgnsq
    :3936) under prefix fx_: yin, expr, wtold, the scalars stepr/acceptr/rejrat/chisqnew and
    the integer arguments with the ran1 state before; wt, wtold, yout, the four returned
    scalars and the ran1 state after."""
    def wrapped(yin, expr, yout, wt, wtold, stepr, acceptr, rejrat, chisqnew, nmin, npt, ncfirst, nterms, nits,
                nfreq):
        if "fx_result" in out:
            return orig(yin, expr, yout, wt, wtold, stepr, acceptr, rejrat, chisqnew, nmin, npt, ncfirst, nterms,
                        nits, nfreq)
        out["fx_yin"] = np.array(yin[: npt + 1], f32)
        out["fx_expr"] = np.array(expr[: npt * nterms + 1], f32)
        out["fx_wtold_in"] = np.array(wtold[: nterms + 1], f32)
        out["fx_scal_in"] = np.array([stepr, acceptr, rejrat, chisqnew], f32)
        out["fx_int"] = np.array([nmin, npt, ncfirst, nterms, nits, nfreq], np.int32)
        for k, v in refstate.ran1_state().items():
            out["fx_ran1_before_" + k] = v
        r = orig(yin, expr, yout, wt, wtold, stepr, acceptr, rejrat, chisqnew, nmin, npt, ncfirst, nterms, nits,
                 nfreq)
        out["fx_wt"] = np.array(wt[: nterms + 1], f32)
        out["fx_wtold"] = np.array(wtold[: nterms + 1], f32)
        out["fx_yout"] = np.array(yout[: npt + 1], f32)
        out["fx_result"] = np.array(r, f32)
        for k, v in refstate.ran1_state().items():
            out["fx_ran1_after_" + k] = v
        return r
    return wrapped


GR_ARRAYS = ("gorintra", "gorinter", "gr2intra", "gr2inter", "entsig")
SQ_ARRAYS = ("soqintra", "soqinter", "sq2intra", "sq2inter")


def capture_sums(common, out, orig_gr, orig_sq):
    """The refinement's sumsq and sumgr calls (epsr_standalone_rev3.py:3642 / :3578, from
    :1637 / :1642) under prefixes ss_ and sg_: the running means and error bars of epsr16 before
    and after ((npairs, points) each), the sample (qwind or wav, (2, npairs, points)), ycoh,
    the real*8 weights fc1, fc2 and the point count."""
    def rows(name, n):
        npairs = int(common.molecom.npairs)
        return np.ascontiguousarray(np.asarray(getattr(common.epsr16, name))[: n + 1, 1:npairs + 1].T, f32)

    def sample(a, n):
        npairs = int(common.molecom.npairs)
        return np.ascontiguousarray(np.asarray(a)[1:3, : n + 1, 1:npairs + 1].transpose(0, 2, 1), f32)

    def take(q, names, n, a, call):
        out[q + "n"] = np.int32(n)
        out[q + "fc"] = np.array([common.sumvalues.fc1, common.sumvalues.fc2], np.float64)
        out[q + "sample"] = sample(a, n)
        out[q + "ycoh"] = np.array(common.epsr16.ycoh[: n + 1], f32)
        for k in names:
            out[q + k + "_in"] = rows(k, n)
        r = call()
        for k in names:
            out[q + k] = rows(k, n)
        return r

    def gr(nz, wav):
        if "sg_n" in out:
            return orig_gr(nz, wav)
        return take("sg_", GR_ARRAYS, int(nz), wav, lambda: orig_gr(nz, wav))

    def sq(nq, qwind):
        if "ss_n" in out:
            return orig_sq(nq, qwind)
        return take("ss_", SQ_ARRAYS, int(nq), qwind, lambda: orig_sq(nq, qwind))
    return gr, sq


GS_EVERY = 20


def capture_gensq(common, out, orig):
    """The refinement's gensq (epsr_standalone_rev3.py:4731, from :1400) under prefix gs_: wav,
    ycoh, n2extr and natomsphere before; and, at every GS_EVERY-th Q point (each point of S(Q)
    depends only on its own column of the sine-transform table), the columns of foqols and the
    intra- and intermolecular S(Q) it wrote."""
    def wrapped(nq, q, sofq, wav):
        if "gs_sel" in out:
            return orig(nq, q, sofq, wav)
        e16, mc = common.epsr16, common.molecom
        npairs, npt1, ntype = int(mc.npairs), int(e16.npt1), int(mc.ntype)
        sel = np.arange(1, int(nq) + 1, GS_EVERY, dtype=np.int32)
        out["gs_sel"] = sel
        out["gs_npt1"] = np.int32(npt1)
        out["gs_wav"] = np.ascontiguousarray(np.asarray(wav)[1:3, : npt1 + 1, 1:npairs + 1].transpose(0, 2, 1), f32)
        out["gs_ycoh"] = np.array(e16.ycoh[: npt1 + 1], f32)
        out["gs_n2extr"] = np.array(mc.n2extr[1:npairs + 1], np.int32) - 1
        out["gs_natomsphere"] = np.array(common.molecom_mod.natomsphere[1:ntype + 1], f32)
        out["gs_foqols"] = np.ascontiguousarray(np.asarray(e16.foqols)[: npt1 + 1, sel].T, f32)
        r = orig(nq, q, sofq, wav)
        out["gs_sofq"] = np.ascontiguousarray(np.asarray(sofq)[1:3, sel, 1:npairs + 1].transpose(0, 2, 1), f32)
        return r
    return wrapped


GE_TABLES = ("xavs", "xavs1", "xavtot", "xavtot1")


def capture_generate_ep(common, out, orig):
    """The refinement's generate_ep call (epsr_standalone_rev3.py:5876, from ptgnsq :4014, the
    program's second) under prefix ge_: the coefficients, weights, grid, tables and scalars it
    reads before; the tables, coefficients, weights, potfac and the basis expgr it wrote after."""
    calls = [0]

    def wrapped(changepotfac):
        calls[0] += 1
        if calls[0] != 2:
            return orig(changepotfac)
        pp, e16, mc = common.potential_par, common.epsr16, common.molecom
        npt, npt2, nterms = int(e16.npt), int(e16.npt2), int(pp.ncoeffp)
        npairs, nsets = int(mc.npairs), int(pp.npairspcof)
        ld = npt + 1
        tab = lambda a: np.ascontiguousarray(np.asarray(a)[:ld, 1:npairs + 1].T, f32)  # noqa: E731
        out["ge_int"] = np.array([npt, npt2, nterms, int(bool(changepotfac))], np.int32)
        out["ge_iref"] = np.array(pp.irefpcof[1:npairs + 1], np.int32) - 1
        out["ge_pcoefp_in"] = np.ascontiguousarray(np.asarray(pp.pcoefp)[: nterms + 1, 1:nsets + 1].T, f32)
        out["ge_pwtold_in"] = np.array(pp.pwtold[: nterms + 1], f32)
        out["ge_scal"] = np.array([common.clustercom.dmax, pp.absolute_energy, pp.erequnit, pp.ereqstep,
                                   pp.potfacamp, pp.potfac], f32)
        out["ge_xstar"] = np.array(e16.xstar[:ld], f32)
        out["ge_wfac"] = np.array(pp.wfac[:ld], f32)
        out["ge_ecoul"] = tab(pp.ecoul)
        for k in GE_TABLES:
            out["ge_" + k + "_in"] = tab(getattr(pp, k))
        r = orig(changepotfac)
        for k in GE_TABLES:
            out["ge_" + k] = tab(getattr(pp, k))
        out["ge_pcoefp"] = np.ascontiguousarray(np.asarray(pp.pcoefp)[: nterms + 1, 1:nsets + 1].T, f32)
        out["ge_pwtold"] = np.array(pp.pwtold[: nterms + 1], f32)
        out["ge_potfac"] = f32(pp.potfac)
        out["ge_expgr"] = np.array(pp.expgr[1: npt2 * nterms + 1], f32)
        return r
    return wrapped


def intra_snapshot(common, out, q):
    """The intramolecular model en_change_intra reads (molecom bond lists, masses, the intra
    reference potential), as the drop-in hands it to the device."""
    mc, cc, pp, e16 = common.molecom, common.clustercom, common.potential_par, common.epsr16
    natom, ntype, npairs = int(mc.natom), int(mc.ntype), int(mc.npairs)
    nb = np.array(mc.nbond[1:natom + 1], np.int32)
    mb = max(1, int(nb.max()) if natom else 1)
    ld = int(e16.npt) + 1
    out[q + "in_nbond"] = nb
    out[q + "in_iabond"] = np.array(mc.iabond)[1:natom + 1, 1:mb + 1].astype(np.int32) - 1
    out[q + "in_tbond"] = np.array(mc.tbond)[1:natom + 1, 1:mb + 1].astype(f32)
    out[q + "in_imageatom"] = np.array(mc.imageatom[1:natom + 1], np.int32) - 1
    out[q + "in_qtype"] = np.array(mc.qtype[1:natom + 1], np.int32)
    out[q + "in_amassa"] = np.array(mc.amassa[1:ntype + 1], f32)
    out[q + "in_amassr"] = np.array(mc.amassr[1:npairs + 1], f32)
    out[q + "in_xav"] = np.ascontiguousarray(np.array(pp.xav)[:ld, 1:npairs + 1].T, f32)
    out[q + "in_xav1"] = np.ascontiguousarray(np.array(pp.xav1)[:ld, 1:npairs + 1].T, f32)
    out[q + "in_scal"] = np.array([f32(e16.cellst) / f32(mc.dmaxmol), mc.sizefactor, mc.tempb, mc.tempang, mc.simt,
                                   float(bool(getattr(mc, "refine_intra", False))),
                                   getattr(mc, "refine_intra_fac", 0.0), mc.tempdih], f32)


def after(common, out, q, result, cos):
    cc, erd = common.clustercom, common.ergpairreference
    nmol, nmt = int(cc.nmol), int(cc.nmoltype)
    mc = common.molecom
    natom = int(mc.natom)
    for k, src, n in (("xa", mc.xa, natom), ("ya", mc.ya, natom), ("za", mc.za, natom), ("xadd", cc.xadd, nmol),
                      ("yadd", cc.yadd, nmol), ("zadd", cc.zadd, nmol)):
        out[q + "after_" + k] = np.array(src[1:n + 1], f32)
    out[q + "after_ergpair"] = np.array(erd.ergpair[1:int(erd.nergpair) + 1], f32)
    for k in ("wholerot", "wholetrans", "internrot", "interntrans"):
        out[q + "after_" + k] = np.array(getattr(cc, k)[1:nmt + 1], f32)
    for k in ("nwhole", "nmovem", "ninter", "nmovei"):
        out[q + "after_" + k] = np.array(getattr(cc, k)[1:3, 1:nmt + 1], np.int32)
    out[q + "after_ergold1"] = f32(erd.ergold[1]) if erd.ergold is not None else f32(0.0)
    out[q + "after_nstepreject"] = np.array(cc.nstepreject[1:nmol + 1], np.int32)
    out[q + "result"] = np.array([result[0], result[1]], f32)
    out[q + "result_nisum"] = np.int32(result[2])
    out[q + "cos"] = np.array(cos, f32)
    for k, v in refstate.ran1_state().items():
        out[q + "ran1_after_" + k] = v


def main():
    src = os.path.join(REF, "EPSR-test")
    work = tempfile.mkdtemp(prefix="epsr_realrun_")
    run = os.path.join(work, "EPSR-test")
    shutil.copytree(src, run)
    prepare_run(run)
    common, program = refstate.load_reference(os.path.join(REF, "src"))
    import importlib
    mods = {"cellneighbourlist": importlib.import_module("epsr26.library.cellneighbourlist"),
            "ato_manipulation_rev4": importlib.import_module("epsr26.library.ato_manipulation_rev4"),
            "molfit": importlib.import_module("epsr26.library.molfit")}
    for name in ("molecom", "clustercom", "epsr16", "potential_par", "lattice", "ran1com", "cellneighbourlist",
                 "ergpairreference", "molecom_mod", "threebody_mod", "coordconstraints_mod", "containerforces_mod"):
        importlib.import_module("epsr26.common." + name)
    common = importlib.import_module("epsr26.common")
    from epsr26.programs import run_program
    molfit = mods["molfit"]
    orig, orig_cos = molfit.molfit, molfit.cosf
    out, state = {}, {"n": 0, "taken": 0}
    rec = []

    def cos_rec(x):
        v = orig_cos(x)
        rec.append(v)
        return v

    def wrapped(fadds, faddbs, nisum, intra, rotfreq, ireset):
        state["n"] += 1
        rot = nisum >= intra or nisum == rotfreq * (nisum // rotfreq)
        if state["n"] not in CAPTURE:
            return orig(fadds, faddbs, nisum, intra, rotfreq, ireset)
        q = "k%d_" % state["taken"]
        snapshot(common, mods, out, q)
        intra_snapshot(common, out, q)
        erd = common.ergpairreference
        out[q + "ergold1"] = f32(erd.ergold[1]) if erd.ergold is not None else f32(0.0)
        out[q + "args"] = np.array([fadds, faddbs], f32)
        out[q + "args_int"] = np.array([nisum, intra, rotfreq, ireset, state["n"]], np.int32)
        rec.clear()
        molfit.cosf = cos_rec
        try:
            r = orig(fadds, faddbs, nisum, intra, rotfreq, ireset)
        finally:
            molfit.cosf = orig_cos
        after(common, out, q, r, rec)
        print(f"captured molfit call {state['n']} (nisum {nisum}, intra {intra}, rotations {rot}) as {q}", flush=True)
        state["taken"] += 1
        if state["taken"] == len(CAPTURE):
            raise _Stop()
        return r

    molfit.molfit = wrapped
    am = mods["ato_manipulation_rev4"]
    cn = mods["cellneighbourlist"]
    orig_cells = cn.initialise_cellneighbourlist
    cn.initialise_cellneighbourlist = capture_cells(common, mods, out, orig_cells)
    orig_atogen, orig_press = am.atogen, am.press
    am.atogen = capture_atogen(common, mods, out, orig_atogen)
    am.press = capture_press(common, mods, out, orig_press)
    orig_fit, orig_ge = program.fit_expansion, program.generate_ep
    program.fit_expansion = capture_fit(common, out, orig_fit)
    program.generate_ep = capture_generate_ep(common, out, orig_ge)
    orig_gs = program.gensq
    program.gensq = capture_gensq(common, out, orig_gs)
    orig_gr, orig_sq = program.sumgr, program.sumsq
    program.sumgr, program.sumsq = capture_sums(common, out, orig_gr, orig_sq)
    cwd = os.getcwd()
    os.chdir(run)
    try:
        run_program("epsr", ["./", "epsr", "200DMSO400Water.EPSR.inp"])
    except _Stop:
        pass
    finally:
        os.chdir(cwd)
        molfit.molfit = orig
        am.atogen, am.press = orig_atogen, orig_press
        cn.initialise_cellneighbourlist = orig_cells
        program.fit_expansion, program.generate_ep = orig_fit, orig_ge
        program.sumgr, program.sumsq = orig_gr, orig_sq
        program.gensq = orig_gs
        shutil.rmtree(work, ignore_errors=True)
    if state["taken"] < len(CAPTURE):
        raise SystemExit("the run ended before molfit call %d" % CAPTURE[-1])
    path = os.path.join(HERE, "realrun.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()
