"""The intramolecular model and moves on the device: en_mole_intra (molfit.py:1327, with
en_atom_intra :923) and the intramolecular cycle of molfit (:124-174, taken when
nisum >= intra), through the C ABI (epsr_en_mole_intra, epsr_molfit_shake).

Atoms are 0-based; bond lists are (natom, maxbond) with the partner atom (-1 unused) and the
bond length in box units (negative: a bond-angle pair, weighted by tempang).
"""

from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib
from ._lib import check

f32 = np.float32


def _p(t):
    return C.c_void_p(t.data_ptr())


def _s():
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


class IntraModel:
    """Device copy of the intramolecular model of one box (epsr_intra_t)."""

    def __init__(self, d, *, nbond, iabond, tbond, amassa, amassr, xav, xav1, stepcl, simt, imageatom=None,
                 qtype=None, ngrot=None, sizefactor=1.0, tempb=1.0, tempang=1.0, refine_intra=False,
                 refine_intra_fac=0.0, dih=None):
        """dih: the rotational groups' dihedral angles, or None -- a dict with grp_nrf, grp_nrl
        (per molecule, 0-based group range), grp_axis (groups x 2 base atoms), grp_dih0 (groups + 1),
        grp_isdih (groups: 1 for DIH), dih_atoms (dihedrals x 2), dih_cos, dih_sin (the host C
        library's cosf/sinf of each angle, as the reference takes them) and tempdih."""
        self.lib = _lib.load(require_device=True)
        self.d = d
        b = d.host
        t = lambda a, dt: torch.from_numpy(np.ascontiguousarray(a, dt)).to(d.dev)  # noqa: E731
        iab = np.asarray(iabond, np.int32)
        self.maxbond = max(1, iab.shape[1] if iab.ndim == 2 else 1)
        pad = lambda a, dt, fill: np.pad(np.asarray(a, dt).reshape(b.natom, -1),  # noqa: E731
                                         ((0, 0), (0, self.maxbond - np.asarray(a).reshape(b.natom, -1).shape[1])),
                                         constant_values=fill)
        self.nbond = t(nbond, np.int32)
        self.iabond = t(pad(iab, np.int32, -1), np.int32)
        self.tbond = t(pad(tbond, f32, 0.0), f32)
        self.imageatom = t(np.full(b.natom, -1, np.int32) if imageatom is None else imageatom, np.int32)
        self.qtype = t(np.zeros(b.natom, np.int32) if qtype is None else qtype, np.int32)
        self.amassa = t(amassa, f32)
        self.amassr = t(amassr, f32)
        ld = b.npt + 1
        self.xav = t(np.asarray(xav, f32)[:, :ld], f32)
        self.xav1 = t(np.asarray(xav1, f32)[:, :ld], f32)
        self.ngrot = t(np.zeros(b.nmol, np.int32) if ngrot is None else ngrot, np.int32)
        s = _lib.Intra()
        s.nbond, s.iabond, s.tbond = _p(self.nbond), _p(self.iabond), _p(self.tbond)
        s.maxbond = self.maxbond
        s.imageatom, s.qtype, s.amassa, s.amassr = _p(self.imageatom), _p(self.qtype), _p(self.amassa), _p(self.amassr)
        s.xav, s.xav1, s.ngrot = _p(self.xav), _p(self.xav1), _p(self.ngrot)
        s.stepcl, s.sizefactor, s.tempb, s.tempang, s.simt = (float(f32(v)) for v in (stepcl, sizefactor, tempb, tempang,
                                                                                       simt))
        s.refine_intra, s.refine_intra_fac = int(bool(refine_intra)), float(f32(refine_intra_fac))
        self.dih = None
        if dih is not None:
            self.dih = {k: t(np.asarray(dih[k]).reshape(-1), np.int32)
                        for k in ("grp_nrf", "grp_nrl", "grp_axis", "grp_dih0", "grp_isdih")}
            na = np.asarray(dih["dih_atoms"], np.int32).reshape(-1)
            self.dih["dih_atoms"] = t(na if na.size else np.zeros(2, np.int32), np.int32)
            for k in ("dih_cos", "dih_sin"):
                v = np.asarray(dih[k], f32).reshape(-1)
                self.dih[k] = t(v if v.size else np.zeros(1, f32), f32)
            for k, v in self.dih.items():
                setattr(s, k, _p(v))
            s.ndih = int(np.asarray(dih["dih_cos"]).size)
            s.tempdih = float(f32(dih["tempdih"]))
        self.c = s

    def en_mole_intra(self, out=None):
        """en_mole_intra of every molecule at the box's current coordinates (device (nmol,))."""
        b = self.d.host
        if out is None:
            out = torch.empty(b.nmol, dtype=torch.float32, device=self.d.dev)
        check(self.lib.epsr_en_mole_intra(C.byref(self.d.cbox), C.byref(self.c), _p(out), _s()))
        return out

    def molfit_shake(self, stepmi, faddbs):
        """One intramolecular cycle of molfit on the box, its pair store and MC state (the
        DeviceBox's mc_setup arrays).  faddbs: device (1,) in/out.  Returns nmovei (device
        (2*nmoltype,): tries, then rejections)."""
        d, b = self.d, self.d.host
        nmovei = torch.zeros(2 * b.nmoltype, dtype=torch.int32, device=d.dev)
        nb = int(self.lib.epsr_molfit_shake_scratch_bytes(b.nmol, b.natom))
        scr = d.scratch("shake", nb)
        check(self.lib.epsr_molfit_shake(C.byref(d.cbox), C.byref(d.store), C.byref(d.cmc), C.byref(self.c),
                                         float(f32(stepmi)), _p(nmovei), _p(faddbs), _p(scr), scr.numel(), _s()))
        return nmovei
