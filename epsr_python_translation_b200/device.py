"""Device-resident state of one EPSR box and the calls of the pair path on it.

``DeviceBox`` owns every device buffer as a PyTorch tensor (coordinates, tables, cell
list, pair-energy store, step sizes, ran1 state) and calls the C ABI of libepsr_gpu.so
with raw pointers.  State stays on the GPU between calls; ``download_*`` copies it back
for host consumers.
"""

from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib
from ._lib import check
from .box import BoxArrays, Ran1State

f32 = np.float32


def _ptr(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


def _stream():
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def press_scalars(nmol, sumc, presst, simt, volume):
    """The closing lines of press (ato_manipulation_rev4.py:4051-4056): the energy per
    molecule in float32 and the pressure in kbar (double arithmetic, stored as float32)."""
    energy = f32(f32(sumc) / f32(nmol))
    pressc = f32(((float(f32(nmol) * f32(simt)) - float(presst) / 3.0) * 100.0)
                 / float(f32(6.0222) * f32(volume)))
    return energy, pressc


def table_cutoff(*tabs) -> int:
    """Last grid index at which any table entry is nonzero (bitwise, so -0 counts)."""
    last = 1
    for t in tabs:
        nz = np.nonzero(np.any(np.ascontiguousarray(t, dtype=f32).view(np.uint32) != 0, axis=0))[0]
        if nz.size:
            last = max(last, int(nz[-1]))
    return last


class DeviceBox:
    def __init__(self, box: BoxArrays, device="cuda"):
        self.lib = _lib.load(require_device=True)
        self.dev = torch.device(device)
        self.host = box
        self.upload(box)
        self.cells = None
        self.store = None
        self._scratch = {}

    # ------------------------------------------------------------------ upload / download
    def _t(self, a, dtype):
        return torch.from_numpy(np.ascontiguousarray(a, dtype=dtype)).to(self.dev)

    def upload(self, b: BoxArrays):
        self.host = b
        d = self
        d.naf = self._t(b.naf, np.int32)
        d.nato = self._t(b.nato, np.int32)
        d.mtype = self._t(b.mtype, np.int32)
        d.itype = self._t(b.itype, np.int32)
        d.xa, d.ya, d.za = (self._t(v, f32) for v in (b.xa, b.ya, b.za))
        d.xadd, d.yadd, d.zadd = (self._t(v, f32) for v in (b.xadd, b.yadd, b.zadd))
        d.pos = torch.zeros(4 * b.natom, dtype=torch.float32, device=self.dev)
        d.npairref = self._t(b.npairref.reshape(-1), np.int32)
        d.n1extr = self._t(b.n1extr, np.int32)
        d.n2extr = self._t(b.n2extr, np.int32)
        d.cfrac = self._t(b.cfrac, f32)
        d.xstar = self._t(b.xstar, f32)
        ld = b.npt + 1
        tab = np.stack([b.xavs, b.xavs1, b.ecoul, b.ecoul1], axis=-1).astype(f32)  # (npairs, ld, 4)
        d.tab = self._t(tab.reshape(-1), f32)
        d.izcut = min(table_cutoff(b.xavs, b.xavs1, b.ecoul, b.ecoul1), b.npt2)
        s = _lib.Box()
        s.nmol, s.natom, s.ntype, s.npairs, s.nmoltype = b.nmol, b.natom, b.ntype, b.npairs, b.nmoltype
        for k in ("naf", "nato", "mtype", "itype", "xa", "ya", "za", "xadd", "yadd", "zadd", "pos", "npairref",
                  "xstar", "tab"):
            setattr(s, k, _ptr(getattr(d, k)))
        s.ld, s.npt2, s.izcut = ld, b.npt2, d.izcut
        s.stepcl = float(b.stepcl)
        s.cubic = 1 if b.cubic else 0
        for i in range(6):
            s.lat[i] = float(b.lat6[i])
        s.maxat = int(np.max(b.nato)) if b.nmol else 0
        self.cbox = s
        check(self.lib.epsr_box_positions(C.byref(s), _stream()))

    def upload_coords(self, xa, ya, za, xadd, yadd, zadd):
        for name, v in (("xa", xa), ("ya", ya), ("za", za), ("xadd", xadd), ("yadd", yadd), ("zadd", zadd)):
            getattr(self, name).copy_(torch.from_numpy(np.ascontiguousarray(v, dtype=f32)))
        check(self.lib.epsr_box_positions(C.byref(self.cbox), _stream()))

    def refresh_positions(self):
        """Recompute the absolute positions after the offset/centre tensors were written."""
        check(self.lib.epsr_box_positions(C.byref(self.cbox), _stream()))

    def minimage_centres(self):
        """The molecule centres put back in the box (runepsr17 after an intramolecular cycle)."""
        check(self.lib.epsr_minimage_centres(C.byref(self.cbox), _stream()))

    def download_coords(self, stream_only=False):
        """Host copies of the coordinates.  stream_only: the box's work was all launched on the
        current stream, so only that stream is waited for (other boxes on other streams keep
        running); otherwise the whole device is synchronised first."""
        if stream_only:
            torch.cuda.current_stream().synchronize()
        else:
            torch.cuda.synchronize()
        return {k: getattr(self, k).cpu().numpy() for k in ("xa", "ya", "za", "xadd", "yadd", "zadd")}

    def scratch(self, name, nbytes):
        t = self._scratch.get(name)
        if t is None or t.numel() < nbytes:
            t = torch.empty(max(int(nbytes), 256), dtype=torch.uint8, device=self.dev)
            self._scratch[name] = t
        return t

    # ------------------------------------------------------------------ ran1
    def ran1_tensor(self, st: Ran1State):
        return self._t(st.as_array(), np.int32)

    def ran1_fill(self, state_t, n):
        out = torch.empty(max(n, 1), dtype=torch.float32, device=self.dev)
        check(self.lib.epsr_ran1_fill(_ptr(state_t), _ptr(out), n, _stream()))
        return out[:n]

    # ------------------------------------------------------------------ cell list
    def _buf(self, name, n, dtype):
        """A persistent device buffer of at least n elements (reallocated only to grow)."""
        t = getattr(self, name, None)
        if t is None or t.numel() < n or t.dtype != dtype:
            t = torch.zeros(max(int(n), 1), dtype=dtype, device=self.dev)
            setattr(self, name, t)
        return t

    def cell_list(self, nmolcell, rmax):
        b = self.host
        dims = np.zeros(4, np.int32)
        lat6 = np.ascontiguousarray(b.lat6, f32)
        lat9 = np.ascontiguousarray(b.lat9, f32)
        check(self.lib.epsr_cell_dims(nmolcell, b.nmol, lat6.ctypes.data_as(C.c_void_p),
                                      dims.ctypes.data_as(C.c_void_p)))
        ncell = int(dims[3])
        c = _lib.Cells()
        self.c_molcellno = self._buf("_c_molcellno", b.nmol, torch.int32)
        self.c_start = self._buf("_c_start", ncell + 1, torch.int32)
        self.c_mols = self._buf("_c_mols", b.nmol, torch.int32)
        self.c_off = self._buf("_c_off", 3 * ncell, torch.int32)
        scr = self._buf("_c_scr", 2 * ncell + 4, torch.int32)
        c.molcellno, c.cell_start, c.cell_mols, c.offsets = (_ptr(t) for t in
                                                             (self.c_molcellno, self.c_start, self.c_mols, self.c_off))
        check(self.lib.epsr_cell_list(_ptr(self.xadd), _ptr(self.yadd), _ptr(self.zadd), b.nmol, nmolcell,
                                      float(f32(rmax)), lat6.ctypes.data_as(C.c_void_p),
                                      lat9.ctypes.data_as(C.c_void_p), C.byref(c), _ptr(scr), scr.numel(), _stream()))
        self.cells = c
        self.nnbrefmax = int(c.nnbrefmax)
        return c

    def download_cells(self):
        torch.cuda.synchronize()
        c = self.cells
        return dict(ncelldiva=c.ncelldiva, ncelldivb=c.ncelldivb, ncelldivc=c.ncelldivc, ncell=c.ncell,
                    ncellneighb=c.ncellneighb, maxcellno=c.maxcellno, molcellno=self.c_molcellno.cpu().numpy(),
                    cell_start=self.c_start.cpu().numpy(), cell_mols=self.c_mols.cpu().numpy(),
                    offsets=self.c_off.cpu().numpy()[: 3 * c.ncellneighb].reshape(-1, 3),
                    nnbrefmax=self.nnbrefmax)

    # ------------------------------------------------------------------ fmolec1
    def fmolec1(self, eintra, strict=True, capacity=None):
        b = self.host
        M = self.nnbrefmax
        cap = capacity or max(100 * b.nmol, 1)
        need = b.nmol + (b.nmol * M) // 2 + 16
        cap = max(cap, min(need, 2**31 - 1))
        st = _lib.Store()
        self.s_nergpairm = self._buf("_s_nergpairm", b.nmol, torch.int32)
        self.s_mol = self._buf("_s_mol", b.nmol * M, torch.int32)
        self.s_ref = self._buf("_s_ref", b.nmol * M, torch.int32)
        self.s_erg = self._buf("_s_erg", cap, torch.float32)
        self.s_n = self._buf("_s_n", 1, torch.int32)
        self.s_mirror = self._buf("_s_mirror", b.nmol * M, torch.int32)
        cap = int(self.s_erg.numel())
        st.mirror = _ptr(self.s_mirror)
        st.nnbrefmax, st.capacity = M, cap
        st.nergpairm, st.molergpair, st.ergpairref, st.ergpair, st.nergpair = (
            _ptr(t) for t in (self.s_nergpairm, self.s_mol, self.s_ref, self.s_erg, self.s_n))
        if isinstance(eintra, torch.Tensor):              # already on the device (epsr_en_mole_intra)
            self.eintra = eintra.to(device=self.dev, dtype=torch.float32).contiguous()
            self._eintra_src = None
        elif getattr(self, "_eintra_src", None) is not eintra:
            self.eintra = self._t(eintra, f32)
            self._eintra_src = eintra
        nb = self.lib.epsr_fmolec1_scratch_bytes(b.nmol, self.cells.ncell, M)
        scr = self.scratch("fmolec1", nb)
        out2 = np.zeros(2, f32)
        check(self.lib.epsr_fmolec1(C.byref(self.cbox), C.byref(self.cells), _ptr(self.eintra), C.byref(st),
                                    _ptr(scr), scr.numel(), 1 if strict else 0, out2.ctypes.data_as(C.c_void_p),
                                    _stream()))
        self.store = st
        return f32(out2[0]), f32(out2[1])

    def download_store(self):
        torch.cuda.synchronize()
        M = self.nnbrefmax
        n = int(self.s_n.item())
        nm = self.host.nmol * M          # the buffers may be larger, kept from a larger region size
        return dict(nnbrefmax=M, nergpair=n, nergpairm=self.s_nergpairm.cpu().numpy(),
                    molergpair=self.s_mol[:nm].cpu().numpy().reshape(-1, M),
                    ergpairref=self.s_ref[:nm].cpu().numpy().reshape(-1, M), ergpair=self.s_erg[:n].cpu().numpy())

    # ------------------------------------------------------------------ molfit
    def mc_setup(self, *, rejrate, stepr, stepm, wholerot, wholetrans, internrot=None, interntrans=None,
                 nstepreject=None, ran1: Ran1State = None, trstepmax, trstepmin, ireset=0, fadds=0.0):
        b = self.host
        nmt = b.nmoltype
        self.m_wholerot = self._t(wholerot, f32)
        self.m_wholetrans = self._t(wholetrans, f32)
        self.m_internrot = self._t(np.zeros(nmt, f32) if internrot is None else internrot, f32)
        self.m_interntrans = self._t(np.zeros(nmt, f32) if interntrans is None else interntrans, f32)
        self.m_nwhole = torch.zeros(2 * nmt, dtype=torch.int32, device=self.dev)
        self.m_nmovem = torch.zeros(2 * nmt, dtype=torch.int32, device=self.dev)
        self.m_nstepreject = self._t(np.zeros(b.nmol, np.int32) if nstepreject is None else nstepreject, np.int32)
        self.m_fadds = self._t(np.array([fadds], f32), f32)
        self.m_ran1 = self.ran1_tensor(ran1 or Ran1State())
        self.m_den = torch.zeros(b.nmol, dtype=torch.float32, device=self.dev)
        self.m_acc = torch.zeros(b.nmol, dtype=torch.int32, device=self.dev)
        m = _lib.Mc()
        m.simt, m.rejrate, m.stepr, m.stepm = float(b.simt), float(f32(rejrate)), float(f32(stepr)), float(f32(stepm))
        m.trstepmax, m.trstepmin, m.ireset = float(trstepmax), float(trstepmin), int(ireset)
        m.wholerot, m.wholetrans, m.internrot, m.interntrans = (
            _ptr(t) for t in (self.m_wholerot, self.m_wholetrans, self.m_internrot, self.m_interntrans))
        m.nwhole, m.nmovem, m.nstepreject, m.fadds, m.ran1 = (
            _ptr(t) for t in (self.m_nwhole, self.m_nmovem, self.m_nstepreject, self.m_fadds, self.m_ran1))
        m.trace_den, m.trace_acc = _ptr(self.m_den), _ptr(self.m_acc)
        m.cos_override = None
        m.strict = 1
        self.m_status = torch.zeros(1, dtype=torch.int32, device=self.dev)
        m.status = _ptr(self.m_status)
        # the next cycle's ran1 values walked on a second stream while a fast cycle runs
        self.m_ahead = torch.zeros(80 + 7 * b.nmol, dtype=torch.int32, device=self.dev)
        m.ahead, m.ahead_cap = _ptr(self.m_ahead), 7 * b.nmol
        self.cmc = m
        return m

    def draws_ahead(self, on=True):
        """Enable or disable the fast path's draws ahead; returns how many cycles took them."""
        m = self.cmc
        m.ahead, m.ahead_cap = (_ptr(self.m_ahead), 7 * self.host.nmol) if on else (None, 0)
        return int(self.m_ahead[2].item())

    def set_rotations(self, intra_model, nrf, nrl, axis, first, last, atoms, stepri=1.0, faddbs=0.0):
        """Internal rotations of rotational groups (type ROT: the dihedral terms of DIH groups
        are not evaluated) before each molecule's whole-molecule move, every rotfreq cycles
        (molfit.py:295-360, rotati :589).  intra_model: intra.IntraModel of this box (its ngrot
        per molecule); nrf/nrl per molecule (0-based group range, nrl < nrf for none); axis
        (groups x 2) axis atoms, rotation about the first; first/last per group into atoms
        (0-based atom indices).  faddbs: the running intramolecular energy change."""
        t = lambda a: self._t(np.asarray(a).reshape(-1), np.int32)  # noqa: E731
        self.r_model = intra_model
        self.r_arrays = [t(nrf), t(nrl), t(axis), t(first), t(last), t(atoms)]
        self.m_ninter = torch.zeros(2 * self.host.nmoltype, dtype=torch.int32, device=self.dev)
        self.m_faddbs = self._t(np.array([faddbs], f32), f32)
        m = self.cmc
        m.intra = C.cast(C.pointer(intra_model.c), C.c_void_p)
        m.rot_nrf, m.rot_nrl, m.rot_axis, m.rot_first, m.rot_last, m.rot_atoms = (_ptr(a) for a in self.r_arrays)
        m.stepri = float(f32(stepri))
        m.ninter, m.faddbs = _ptr(self.m_ninter), _ptr(self.m_faddbs)

    def set_cos_override(self, cos_override=None):
        """Cosines the next MC cycle uses in draw order instead of its own (a test hook that
        proves the chain bit for bit against the reference's cosf values); None: its own."""
        self._cos = None
        if cos_override is not None:
            self._cos = self._t(cos_override, f32)
            self.cmc.cos_override = _ptr(self._cos)
        else:
            self.cmc.cos_override = None

    def molfit(self, strict=True, cos_override=None, rotcycle=True):
        b = self.host
        if int(np.max(b.nato)) > 64:
            raise _lib.EpsrGpuError(4, "molfit: molecules of more than 64 atoms are not supported")
        m = self.cmc
        m.strict = 1 if strict else 0
        m.rotcycle = 1 if rotcycle else 0
        self.set_cos_override(cos_override)
        nb = self.lib.epsr_molfit_scratch_bytes(b.nmol, b.natom, self.nnbrefmax)
        scr = self.scratch("molfit", nb)
        check(self.lib.epsr_molfit(C.byref(self.cbox), C.byref(self.cells), C.byref(self.store), C.byref(m), _ptr(scr),
                                   scr.numel(), _stream()))

    def check_status(self):
        """Raise if a molfit cycle reported an error (synchronises)."""
        v = int(self.m_status.item())
        if v:
            raise _lib.EpsrGpuError(4 if v == 1 else 5, {1: "molecule larger than 64 atoms",
                                                         2: "fast-path resolver timed out"}.get(v, str(v)))

    def download_mc(self):
        torch.cuda.synchronize()
        nmt = self.host.nmoltype
        return dict(wholerot=self.m_wholerot.cpu().numpy(), wholetrans=self.m_wholetrans.cpu().numpy(),
                    internrot=self.m_internrot.cpu().numpy(), interntrans=self.m_interntrans.cpu().numpy(),
                    nwhole=self.m_nwhole.cpu().numpy().reshape(2, nmt), nmovem=self.m_nmovem.cpu().numpy().reshape(2, nmt),
                    nstepreject=self.m_nstepreject.cpu().numpy(), fadds=f32(self.m_fadds.cpu().numpy()[0]),
                    ran1=Ran1State.from_array(self.m_ran1.cpu().numpy()), den=self.m_den.cpu().numpy(),
                    acc=self.m_acc.cpu().numpy())

    # ------------------------------------------------------------------ atogen
    def atogen(self, ngrsamples, ran1_t, rminex, ycoh=None, sizefactor=1.0, npt1=None):
        b = self.host
        npt1 = b.npt1 if npt1 is None else npt1
        ld = b.npt + 1
        self.a_wav = torch.zeros(2 * b.npairs * ld, dtype=torch.float32, device=self.dev)
        self.a_potex = torch.zeros(b.npairs, dtype=torch.float32, device=self.dev)
        counts = self.scratch("atogen_counts", 8 * (2 * b.npairs * ld + b.npairs))
        # device tensors are used as given (no upload per call); host arrays are copied
        if isinstance(rminex, torch.Tensor):
            self.a_rminex = rminex
        else:
            self.a_rminex = self._t(rminex, f32)
        if isinstance(ycoh, torch.Tensor):
            self.a_ycoh = ycoh
        else:
            self.a_ycoh = self._t(np.zeros(ld, f32) if ycoh is None else np.asarray(ycoh, f32)[:ld], f32)
        nb = self.lib.epsr_atogen_scratch_bytes(b.nmol, b.natom, b.nmoltype, b.ntype)
        scr = self.scratch("atogen", nb)
        ngr = np.array([ngrsamples], np.int32)
        check(self.lib.epsr_atogen(C.byref(self.cbox), npt1, float(sizefactor), float(b.dmax), _ptr(self.a_rminex),
                                   _ptr(self.cfrac), _ptr(self.a_ycoh), _ptr(self.n1extr), _ptr(self.n2extr), b.natomr,
                                   ngr.ctypes.data_as(C.c_void_p), _ptr(ran1_t), _ptr(self.a_wav), ld,
                                   _ptr(self.a_potex), _ptr(counts), _ptr(scr), scr.numel(), _stream()))
        self.last_pair_updates = int(self.lib.epsr_atogen_last_pair_updates())
        return int(ngr[0])

    # ------------------------------------------------------------------ press
    def press(self, npt1=None, strict=True):
        """press ato_manipulation_rev4.py:3903-4062 on the current store: returns (sumc,
        presst) -- the float32 energy sum and the double virial sum over the stored pairs."""
        b = self.host
        npt1 = b.npt1 if npt1 is None else npt1
        nb = self.lib.epsr_press_scratch_bytes(b.nmol, self.nnbrefmax)
        scr = self.scratch("press", nb)
        sums = np.zeros(2, np.float64)
        check(self.lib.epsr_press(C.byref(self.cbox), C.byref(self.store), int(npt1), _ptr(scr), scr.numel(),
                                  1 if strict else 0, sums.ctypes.data_as(C.c_void_p), _stream()))
        return f32(sums[0]), float(sums[1])

    def download_wav(self):
        torch.cuda.synchronize()
        b = self.host
        return self.a_wav.cpu().numpy().reshape(2, b.npairs, b.npt + 1), self.a_potex.cpu().numpy()
