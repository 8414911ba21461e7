"""A stand-in for the device layer of the drop-in (device.DeviceBox, intra.IntraModel) whose
every routine is the oracle's C restatement on the host: test infrastructure, so that the
drop-in's own host side -- reading the COMMON blocks, the cell list and pair store written
back into them, the routing of molfit by nisum, the ran1 state in and out, the step arrays
and counters written back -- runs inside the reference's unchanged epsr loop on a machine
without a GPU.  Every routine the drop-in installs by default has its stand-in: the cell
list, fmolec1 and molfit (the intramolecular cycle with rotational groups included), atogen,
press, gensq, the running sums, stog, fit_expansion and generate_ep; the host-side library
routines (the EP basis, generate_rp) run as they are.  The device layer itself is checked
against the same oracle by the GPU tests.  ``install(monkeypatch)`` puts them in place.

The state the device would hold (coordinates, cells, pair store, MC arrays) is held here as
NumPy arrays and CPU tensors with the device layer's names and layouts (the drop-in reads and
writes the store tensors directly)."""

from __future__ import annotations

import copy
import types

import numpy as np
import torch

from epsr_python_translation_b200.box import BoxArrays, Ran1State
from oracle import oracle

f32 = np.float32
COORDS = ("xa", "ya", "za", "xadd", "yadd", "zadd")


def _copy_box(b: BoxArrays) -> BoxArrays:
    return copy.deepcopy(b)


class OracleDeviceBox:
    """device.DeviceBox's interface over the oracle (see the module docstring).  ``journal``:
    when a list, every box made appends "box" and then each routine it runs to it."""

    journal = None

    def __init__(self, b, device=None):
        self.dev = "cpu"
        self.host = b
        self.box = _copy_box(b)
        self.cells = None
        self.nnbrefmax = 0
        self.cmc = None
        self.r = None
        self._cos = None
        self.calls = [] if OracleDeviceBox.journal is None else OracleDeviceBox.journal
        self.calls.append("box")

    # ------------------------------------------------------------------ state in and out
    def upload(self, b):
        self.host = b
        self.box = _copy_box(b)

    def upload_coords(self, xa, ya, za, xadd, yadd, zadd):
        for k, v in zip(COORDS, (xa, ya, za, xadd, yadd, zadd)):
            setattr(self.box, k, np.array(v, f32))

    def download_coords(self, stream_only=False):
        return {k: np.array(getattr(self.box, k), f32) for k in COORDS}

    def ran1_tensor(self, st: Ran1State):
        return torch.from_numpy(st.as_array().copy())

    # ------------------------------------------------------------------ cells
    def cell_list(self, nmolcell, rmax):
        self.calls.append("cell_list")
        self.cells = oracle.cell_list(self.box, int(nmolcell), f32(rmax))
        self.nnbrefmax = int(self.cells["nnbrefmax"])
        return self.cells

    def download_cells(self):
        c = self.cells
        nb = int(c["ncellneighb"])
        off = np.stack([np.asarray(c[k])[:nb] for k in ("ia_off", "ib_off", "ic_off")], 1).astype(np.int32)
        return dict(ncelldiva=c["ncelldiva"], ncelldivb=c["ncelldivb"], ncelldivc=c["ncelldivc"], ncell=c["ncell"],
                    ncellneighb=nb, maxcellno=c["maxcellno"], molcellno=np.array(c["molcellno"]),
                    cell_start=np.array(c["cell_start"]), cell_mols=np.array(c["cell_mols"]), offsets=off,
                    nnbrefmax=self.nnbrefmax)

    # ------------------------------------------------------------------ pair store
    def fmolec1(self, eintra, strict=True, capacity=None):
        self.calls.append("fmolec1")
        st = oracle.fmolec1(self.box, self.cells, np.asarray(eintra, f32), capacity)
        self.s_nergpairm = torch.from_numpy(np.ascontiguousarray(st["nergpairm"], np.int32))
        self.s_mol = torch.from_numpy(np.ascontiguousarray(st["molergpair"], np.int32).reshape(-1))
        self.s_ref = torch.from_numpy(np.ascontiguousarray(st["ergpairref"], np.int32).reshape(-1))
        self.s_erg = torch.from_numpy(np.ascontiguousarray(st["ergpair"], f32))
        self.s_n = torch.tensor([int(st["nergpair"])], dtype=torch.int32)
        return f32(st["ftest"]), f32(st["ftestb"])

    def _store(self):
        """The store as the oracle takes it: views of the tensors, so its updates land there."""
        nm = self.host.nmol * self.nnbrefmax
        return dict(nnbrefmax=self.nnbrefmax, nergpair=int(self.s_n[0]), nergpairm=self.s_nergpairm.numpy(),
                    molergpair=self.s_mol.numpy()[:nm], ergpairref=self.s_ref.numpy()[:nm], ergpair=self.s_erg.numpy())

    def download_store(self):
        M, n = self.nnbrefmax, int(self.s_n[0])
        nm = self.host.nmol * M
        return dict(nnbrefmax=M, nergpair=n, nergpairm=self.s_nergpairm.numpy().copy(),
                    molergpair=self.s_mol.numpy()[:nm].reshape(-1, M).copy(),
                    ergpairref=self.s_ref.numpy()[:nm].reshape(-1, M).copy(), ergpair=self.s_erg.numpy()[:n].copy())

    # ------------------------------------------------------------------ molfit
    def mc_setup(self, *, rejrate, stepr, stepm, wholerot, wholetrans, internrot=None, interntrans=None,
                 nstepreject=None, ran1=None, trstepmax, trstepmin, ireset=0, fadds=0.0):
        nmt = self.host.nmoltype
        self.mc = dict(rejrate=f32(rejrate), stepr=f32(stepr), stepm=f32(stepm), ireset=int(ireset),
                       wholerot=np.array(wholerot, f32), wholetrans=np.array(wholetrans, f32),
                       internrot=np.array(internrot, f32), interntrans=np.array(interntrans, f32),
                       nstepreject=np.array(nstepreject, np.int32), nwhole=np.zeros(2 * nmt, np.int32),
                       nmovem=np.zeros(2 * nmt, np.int32))
        self.m_fadds = f32(fadds)
        self.m_ran1 = self.ran1_tensor(ran1 or Ran1State())
        self.r = None
        self.cmc = types.SimpleNamespace(ran1=None, cos_override=None)
        return self.cmc

    def set_rotations(self, intra_model, nrf, nrl, axis, first, last, atoms, stepri=1.0, faddbs=0.0):
        self.r = dict(model=intra_model.m, nrf=np.asarray(nrf, np.int32), nrl=np.asarray(nrl, np.int32),
                      axis=np.asarray(axis, np.int32).reshape(-1), first=np.asarray(first, np.int32),
                      last=np.asarray(last, np.int32), atoms=np.asarray(atoms, np.int32), stepri=f32(stepri),
                      faddbs=f32(faddbs))
        self.mc["ngrot"] = np.asarray(intra_model.m["ngrot"], np.int32)
        self.m_ninter = torch.zeros(2 * self.host.nmoltype, dtype=torch.int32)
        self.m_faddbs = torch.tensor([float(f32(faddbs))], dtype=torch.float32)

    def set_cos_override(self, cos_override=None):
        if cos_override is not None:
            raise NotImplementedError("the oracle stand-in draws its own cosines")

    def _ran1(self):
        return Ran1State.from_array(self.m_ran1.numpy())

    def _ran1_back(self, st):
        self.m_ran1.copy_(torch.from_numpy(st.as_array()))

    def molfit(self, strict=True, cos_override=None, rotcycle=True):
        self.calls.append("molfit")
        self.set_cos_override(cos_override)
        rot = None
        if self.r is not None:
            rot = dict(self.r, rotcycle=1 if rotcycle else 0)
        fa, tr, ran1 = oracle.molfit(self.box, self.cells, self._store(), self.mc, self._ran1(), self.m_fadds,
                                     record_cos=False, rot=rot)
        self.m_fadds = f32(fa)
        self._ran1_back(ran1)
        if rot is not None:
            self.m_ninter.copy_(torch.from_numpy(tr["ninter"]))
            self.m_faddbs[0] = float(tr["faddbs"])

    def check_status(self):
        return None

    def download_mc(self):
        nmt = self.host.nmoltype
        m = self.mc
        return dict(wholerot=m["wholerot"].copy(), wholetrans=m["wholetrans"].copy(),
                    internrot=m["internrot"].copy(), interntrans=m["interntrans"].copy(),
                    nwhole=m["nwhole"].reshape(2, nmt).copy(), nmovem=m["nmovem"].reshape(2, nmt).copy(),
                    nstepreject=m["nstepreject"].copy(), fadds=f32(self.m_fadds), ran1=self._ran1())

    # ------------------------------------------------------------------ atogen, press
    def atogen(self, ngrsamples, ran1_t, rminex, ycoh=None, sizefactor=1.0, npt1=None):
        self.calls.append("atogen")
        wav, potex, n, ran1 = oracle.atogen(self.box, int(ngrsamples), Ran1State.from_array(ran1_t.numpy()),
                                            np.asarray(rminex, f32), ycoh, f32(sizefactor))
        ran1_t.copy_(torch.from_numpy(ran1.as_array()))
        self._wav = (wav, potex)
        return n

    def download_wav(self):
        return self._wav

    def press(self, npt1=None, strict=True):
        """(sumc, presst) of the stored pairs; the caller forms the energy and pressure from
        them with the box volume, so the oracle's own scalars (volume 1 here) go unused."""
        self.calls.append("press")
        r = oracle.press(self.box, self._store(), int(npt1), self.box.simt, 1.0)
        return f32(r["sumc"]), float(r["presst"])


class OracleIntraModel:
    """intra.IntraModel's interface over the oracle: ``m`` is the oracle's model dict."""

    def __init__(self, d, *, nbond, iabond, tbond, amassa, amassr, xav, xav1, stepcl, simt, imageatom=None,
                 qtype=None, ngrot=None, sizefactor=1.0, tempb=1.0, tempang=1.0, refine_intra=False,
                 refine_intra_fac=0.0, dih=None):
        b = d.host
        self.d = d
        self.m = dict(nbond=nbond, iabond=iabond, tbond=tbond, amassa=amassa, amassr=amassr, xav=xav, xav1=xav1,
                      stepcl=f32(stepcl), simt=f32(simt), sizefactor=f32(sizefactor), tempb=f32(tempb),
                      tempang=f32(tempang), refine_intra=bool(refine_intra), refine_intra_fac=f32(refine_intra_fac),
                      imageatom=np.full(b.natom, -1, np.int32) if imageatom is None else imageatom,
                      qtype=np.zeros(b.natom, np.int32) if qtype is None else qtype,
                      ngrot=np.zeros(b.nmol, np.int32) if ngrot is None else ngrot, dih=dih)

    def en_mole_intra(self, out=None):
        self.d.calls.append("en_mole_intra")
        return oracle.en_mole_intra_all(self.d.box, self.m)

    def molfit_shake(self, stepmi, faddbs):
        """The intramolecular cycle; faddbs: (1,) tensor in/out; returns nmovei (2*nmoltype,).
        The work array's first slot starts at 0, as on the device."""
        d = self.d
        d.calls.append("molfit_shake")
        fb = f32(faddbs[0].item())
        if d.r is not None:
            rot = dict(d.r, model=self.m)
            fa, fb, nmovei, ninter, _, ran1, _ = oracle.molfit_shake_rot(d.box, d._store(), d.mc, rot, f32(stepmi),
                                                                          d._ran1(), d.m_fadds, fb, 0.0)
            d.m_ninter.copy_(torch.from_numpy(ninter))
        else:
            fa, fb, nmovei, _, ran1 = oracle.molfit_shake(d.box, d._store(), d.mc, self.m, f32(stepmi), d._ran1(),
                                                          d.m_fadds, fb, 0.0)
        d.m_fadds = f32(fa)
        d._ran1_back(ran1)
        faddbs[0] = float(fb)
        return torch.from_numpy(np.asarray(nmovei, np.int32))


# ---------------------------------------------------------------------- transforms and the EP
def _note(name):
    j = OracleDeviceBox.journal
    if j is not None:
        j.append(name)


def gensq(nq, npt1, wav, ldw, foqols, sj, si, ycoh, n2extr, natomsphere, npairs):
    """transforms.gensq over the oracle (foqols (r points, Q points), strides (nq+1, 1))."""
    _note("gensq")
    fq = np.asarray(foqols, f32)
    assert fq.ndim == 2 and (sj, si) == (fq.shape[1], 1)
    out = oracle.gensq(int(nq), int(npt1), wav.numpy().reshape(2, npairs, ldw), np.ascontiguousarray(fq.T),
                       np.asarray(ycoh, f32), np.asarray(n2extr, np.int32), np.asarray(natomsphere, f32))
    return torch.from_numpy(out.reshape(-1))


def sumgr(nz, wav, ycoh, fc1, fc2, acc):
    """transforms.sumgr over the oracle: acc updated in place."""
    from epsr_python_translation_b200.transforms import GR_ARRAYS
    _note("sumgr")
    npairs, ldw = acc["gorintra"].shape
    out = oracle.sumgr(int(nz), wav.numpy().reshape(2, npairs, ldw), ycoh.numpy(), fc1, fc2,
                       {k: acc[k].numpy() for k in GR_ARRAYS})
    for k in GR_ARRAYS:
        acc[k].copy_(torch.from_numpy(out[k]))
    return acc


def sumsq(nq, qwind, fc1, fc2, acc):
    """transforms.sumsq over the oracle: acc updated in place."""
    from epsr_python_translation_b200.transforms import SQ_ARRAYS
    _note("sumsq")
    npairs, ldq = acc["soqintra"].shape
    out = oracle.sumsq(int(nq), qwind.numpy().reshape(2, npairs, ldq), fc1, fc2, {k: acc[k].numpy() for k in SQ_ARRAYS})
    for k in SQ_ARRAYS:
        acc[k].copy_(torch.from_numpy(out[k]))
    return acc


def stog(rho, q, sofq_pairs, r, nqmin, nqmax, xwt):
    """transforms.stog over the oracle: (npairs, nr+1)."""
    _note("stog")
    sp = sofq_pairs.numpy() if isinstance(sofq_pairs, torch.Tensor) else np.asarray(sofq_pairs, f32)
    return torch.from_numpy(oracle.stog(f32(rho), np.asarray(q, f32), sp, np.asarray(r, f32), nqmin, nqmax, xwt))


def fit_expansion(yin, expr, wtold, stepr, nmin, npt, ncfirst, nterms, nits, nfreq, ran1_t, acceptr=0.0, rejrat=0.0,
                  chisqnew=0.0, strict=True):
    """transforms.fit_expansion over the oracle (strict: the reference's float sums)."""
    _note("fit_expansion")
    res, ran1 = oracle.fit_expansion(np.asarray(yin, f32), np.asarray(expr, f32), np.asarray(wtold, f32), f32(stepr),
                                     int(nmin), int(npt), int(ncfirst), int(nterms), int(nits), int(nfreq),
                                     Ran1State.from_array(ran1_t.numpy()), fast=not strict, acceptr=f32(acceptr),
                                     rejrat=f32(rejrat), chisqnew=f32(chisqnew))
    ran1_t.copy_(torch.from_numpy(ran1.as_array()))
    return dict(wt=torch.from_numpy(res["wt"]), wtold=torch.from_numpy(res["wtold"]), yout=torch.from_numpy(res["yout"]),
                stepr=f32(res["stepr"]), acceptr=f32(res["acceptr"]), rejrat=f32(res["rejrat"]), chisq=f32(res["chisq"]),
                trials=res["trials"])


def generate_ep(npt, npt2, nterms, expgr, pcoefp, iref, dmax, xstar, wfac, ecoul, tabs, pwtold, absolute_energy,
                erequnit, ereqstep, potfacamp, potfac, changepotfac=True, result=None):
    """potential.generate_ep over the oracle: tabs, pcoefp, pwtold and potfac updated in place."""
    _note("generate_ep")
    out, pc, pw, pf, energabs, pressfac = oracle.generate_ep(
        int(npt), int(npt2), int(nterms), expgr.numpy(), pcoefp.numpy(), np.asarray(iref, np.int32), f32(dmax),
        xstar.numpy(), wfac.numpy(), ecoul.numpy(), {k: t.numpy() for k, t in tabs.items()}, pwtold.numpy(),
        np.array([absolute_energy, erequnit, ereqstep, potfacamp], f32), f32(potfac.numpy()[0]), bool(changepotfac))
    for k, t in tabs.items():
        t.copy_(torch.from_numpy(out[k]))
    pcoefp.copy_(torch.from_numpy(pc))
    pwtold.copy_(torch.from_numpy(pw))
    potfac[0] = float(pf)
    return torch.tensor([float(energabs), float(pressfac)], dtype=torch.float32)


def install(monkeypatch):
    """Put the stand-ins in place of the device layer for the rest of a test."""
    from epsr_python_translation_b200 import _lib, device, intra, potential, transforms
    real_load = _lib.load
    monkeypatch.setattr(device, "DeviceBox", OracleDeviceBox)
    monkeypatch.setattr(intra, "IntraModel", OracleIntraModel)
    for name in ("gensq", "sumgr", "sumsq", "stog", "fit_expansion"):
        monkeypatch.setattr(transforms, name, globals()[name])
    monkeypatch.setattr(potential, "generate_ep", generate_ep)
    monkeypatch.setattr(_lib, "load", lambda require_device=False: real_load())
    monkeypatch.setattr(torch.cuda, "synchronize", lambda *a, **k: None)
    monkeypatch.setattr(torch.Tensor, "cuda", lambda self, *a, **k: self)
    monkeypatch.setattr(OracleDeviceBox, "journal", [])
    return OracleDeviceBox.journal
