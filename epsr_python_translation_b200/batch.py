"""Many independent boxes advanced together on the device (csrc/batch.cu).

``BatchBoxes`` packs any number of cubic boxes of uneven size and composition (configs.System)
into one set of device arrays and runs the checkerboard Metropolis scheme over all of them at
once: one propose and one decide launch per step for every box together (plus the surrogate
network's two launches with delayed acceptance), the steps of a sweep captured in one CUDA
graph.  The sampled distribution is the reference method's -- the same tabulated pair energies
(molfit.py:1251-1279), temperature and Metropolis test (molfit.py:401-408) -- only the order in
which molecules are visited and the proposal differ (see csrc/batch.cu).

Per box the cell grid is chosen here: ncell cells a side coloured with stride^3 colours such
that (stride - 1) cells cover the interaction range (the table cutoff plus twice the largest
molecular radius), maximising the moves made in parallel, (ncell/stride)^3.
"""

from __future__ import annotations

import ctypes as C
import math

import numpy as np
import torch

from . import _lib
from ._lib import check

f32 = np.float32
FEAT_IN = 1280
FEAT_RMAX_A = 8.0
FIRST_LETTER_CLASS = {"S": 0, "C": 1, "N": 1, "O": 2, "H": 3}


def element_class(label):
    """Feature class of an atom label by its element: S and Si 0, C and N 1, O 2, H 3 (others 1);
    the ten unordered class pairs are the features' pair types."""
    if label.startswith("Si"):
        return 0
    return FIRST_LETTER_CLASS.get(label[:1].upper(), 1)


class BoxDesc(C.Structure):
    _fields_ = [("mol0", C.c_int32), ("nmol", C.c_int32), ("atom0", C.c_int32), ("natom", C.c_int32),
                ("ncell", C.c_int32), ("stride", C.c_int32), ("cell0", C.c_int32), ("slot0", C.c_int32),
                ("nslot", C.c_int32), ("tab0", C.c_int32), ("ld", C.c_int32), ("izcut", C.c_int32),
                ("npairref0", C.c_int32), ("ntype", C.c_int32), ("xstar0", C.c_int32), ("nrange", C.c_int32),
                ("nrange_feat", C.c_int32), ("stepcl", C.c_float), ("beta", C.c_float), ("dmax", C.c_float),
                ("rint", C.c_float), ("rfeat", C.c_float), ("rfeat_c", C.c_float), ("rotmax", C.c_float),
                ("transmax", C.c_float),
                ("key0", C.c_uint32), ("key1", C.c_uint32), ("shift", C.c_float * 3), ("colour_off", C.c_int32),
                ("sweep", C.c_int64)]


class Bmc(C.Structure):
    _fields_ = [("nbox", C.c_int32), ("nmol", C.c_int32), ("natom", C.c_int32), ("ncell", C.c_int32),
                ("nslot", C.c_int32), ("threads", C.c_int32), ("box", C.c_void_p), ("slot_box", C.c_void_p), ("mol_box", C.c_void_p),
                ("naf", C.c_void_p), ("nato", C.c_void_p), ("fclass", C.c_void_p), ("xa", C.c_void_p),
                ("ya", C.c_void_p), ("za", C.c_void_p), ("xadd", C.c_void_p), ("yadd", C.c_void_p),
                ("zadd", C.c_void_p), ("pos", C.c_void_p), ("tab", C.c_void_p), ("xstar", C.c_void_p),
                ("npairref", C.c_void_p), ("cell_start", C.c_void_p), ("cell_mols", C.c_void_p),
                ("mol_cell", C.c_void_p), ("slot_mol", C.c_void_p), ("slot_new", C.c_void_p),
                ("slot_off", C.c_void_p), ("slot_centre", C.c_void_p), ("energy", C.c_void_p),
                ("emol", C.c_void_p), ("counters", C.c_void_p), ("sweep_counter", C.c_void_p),
                ("status", C.c_void_p)]


class BmcHist(C.Structure):
    _fields_ = [("nitems", C.c_int32), ("tile", C.c_int32), ("max_bins", C.c_int32), ("items", C.c_void_p),
                ("hist0", C.c_void_p), ("wav0", C.c_void_p), ("npairs", C.c_void_p), ("npt1", C.c_void_p),
                ("ldw", C.c_void_p), ("pair0", C.c_void_p), ("type0", C.c_void_p), ("n1extr", C.c_void_p),
                ("n2extr", C.c_void_p), ("atom_mol", C.c_void_p), ("rminex", C.c_void_p), ("cfrac", C.c_void_p),
                ("csampled", C.c_void_p), ("counts", C.c_void_p), ("wav", C.c_void_p), ("potex", C.c_void_p),
                ("pairs", C.c_void_p)]


def _p(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


def _stream():
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def choose_grid(R, transmax, max_stride=8):
    """(stride, ncell) maximising the parallel moves (ncell/stride)^3 subject to
    (stride - 1)/ncell >= R (box units) and ncell a multiple of stride; cells at least four
    maximum displacements wide where possible (so few moves leave their cell).  Ties go to
    the smaller stride.  None if the box is too small for any colouring."""
    best = None
    for s in range(2, max_stride + 1):
        m = 1
        while True:
            n = s * m
            if (s - 1) / n < R:
                break
            m += 1
        m -= 1
        if m < 1:
            continue
        n = s * m
        key = (m ** 3, 1.0 / n >= 4 * transmax, -s)
        if best is None or key > best[0]:
            best = (key, s, n)
    return None if best is None else (best[1], best[2])


def value_cutoff(*tabs):
    """Last grid index at which any table entry is nonzero in value (a -0 entry adds nothing to
    an energy, so the interaction range ends before it)."""
    last = 1
    for t in tabs:
        nz = np.nonzero(np.any(np.asarray(t, np.float32) != 0, axis=0))[0]
        if nz.size:
            last = max(last, int(nz[-1]))
    return last


def partition_boxes(natoms, world):
    """Boxes split over `world` GPUs, greedily by atom count (the largest box next onto the
    least-loaded rank): returns per rank the list of box indices, each in ascending order.
    The boxes are independent, so the ranks need no exchange during a sweep."""
    load = [0] * world
    parts = [[] for _ in range(world)]
    for i in sorted(range(len(natoms)), key=lambda k: (-natoms[k], k)):
        r = min(range(world), key=lambda q: (load[q], q))
        parts[r].append(i)
        load[r] += natoms[i]
    return [sorted(p) for p in parts]


def molecular_radius(s):
    """Largest distance of an atom from its molecule's centre (box units)."""
    r = np.sqrt(s.xa.astype(np.float64) ** 2 + s.ya.astype(np.float64) ** 2 + s.za.astype(np.float64) ** 2)
    return float(np.max(r)) if r.size else 0.0


class BatchBoxes:
    def __init__(self, systems, rot_deg=10.0, trans_A=0.5, seed=1, device="cuda"):
        self.lib = _lib.load(require_device=True)
        self.dev = torch.device(device)
        self.systems = list(systems)
        descs, tabs, xstars, prs = [], [], [], []
        mol0 = atom0 = cell0 = slot0 = tab0 = xs0 = pr0 = 0
        naf, nato, fclass, itype = [], [], [], []
        xa, ya, za, xadd, yadd, zadd = [], [], [], [], [], []
        slot_box, mol_box, cell_box = [], [], []
        self.grid = []
        for b, s in enumerate(self.systems):
            d = BoxDesc()
            L = float(s.L)
            dmax = float(s.dmax)
            ld = s.grid["npt"] + 1
            izcut = min(value_cutoff(s.xavs, s.xavs1, s.ecoul, s.ecoul1), int(s.grid["npt2"]))
            stepcl = f32(s.cellst) / f32(s.dmax)
            rc = (izcut + 1) * float(stepcl)          # no table entry beyond this distance (box units)
            rext = molecular_radius(s)
            transmax = trans_A / L
            R = rc + 2.0 * rext
            g = choose_grid(R, transmax)
            if g is None:
                raise _lib.EpsrGpuError(1, f"box {b} ({s.name}, L = {L:.1f} A) is too small for a colouring")
            stride, ncell = g
            self.grid.append((stride, ncell))
            d.mol0, d.nmol, d.atom0, d.natom = mol0, s.nmol, atom0, s.natom
            d.ncell, d.stride, d.cell0, d.slot0 = ncell, stride, cell0, slot0
            d.nslot = (ncell // stride) ** 3
            d.tab0, d.ld, d.izcut, d.npairref0, d.ntype, d.xstar0 = tab0, ld, izcut, pr0, s.ntype, xs0
            d.nrange = int(math.ceil(R * ncell))
            d.nrange_feat = int(math.ceil((FEAT_RMAX_A / dmax + 2.0 * rext) * ncell))
            d.stepcl, d.beta, d.dmax = float(stepcl), float(f32(1.0) / f32(s.simt)), dmax
            d.rint = R + math.sqrt(3.0) * transmax + 1e-6
            d.rfeat = FEAT_RMAX_A / dmax
            d.rfeat_c = d.rfeat + 2.0 * rext + math.sqrt(3.0) * transmax + 1e-6
            d.rotmax, d.transmax = math.radians(rot_deg), transmax
            d.key0 = (0x9E3779B1 * (seed + 1) + 0x7F4A7C15 * b) & 0xFFFFFFFF
            d.key1 = (0x85EBCA6B * (b + 1) ^ (seed * 0xC2B2AE35)) & 0xFFFFFFFF
            descs.append(d)
            tab = np.stack([s.xavs, s.xavs1, s.ecoul, s.ecoul1], axis=-1).astype(f32)
            tabs.append(tab.reshape(-1, 4))
            xstars.append(s.xstar.astype(f32))
            prs.append(s.npairref.reshape(-1).astype(np.int32))
            naf.append(s.naf + atom0)
            nato.append(s.nato)
            itype.append(s.itype)
            fclass.append(np.array([element_class(s.type_labels[t]) for t in s.itype], np.int32))
            xa.append(s.xa), ya.append(s.ya), za.append(s.za)
            xadd.append(s.xadd), yadd.append(s.yadd), zadd.append(s.zadd)
            slot_box.append(np.full(d.nslot, b, np.int32))
            mol_box.append(np.full(s.nmol, b, np.int32))
            cell_box.append(np.full(ncell ** 3, b, np.int32))
            mol0 += s.nmol
            atom0 += s.natom
            cell0 += ncell ** 3
            slot0 += d.nslot
            tab0 += tab.shape[0] * tab.shape[1]
            xs0 += s.xstar.shape[0]
            pr0 += s.ntype * s.ntype
        self.nbox, self.nmol, self.natom, self.ncell, self.nslot = len(descs), mol0, atom0, cell0, slot0
        self.descs = descs
        self.steps_per_sweep = max(int(math.ceil(d.nmol / d.nslot)) for d in descs)
        t = lambda a, dt: torch.from_numpy(np.ascontiguousarray(np.concatenate(a), dtype=dt)).to(self.dev)  # noqa
        self.box_t = torch.from_numpy(np.frombuffer(bytes(b"".join(bytes(d) for d in descs)), np.uint8).copy()).to(
            self.dev)
        self.slot_box = t(slot_box, np.int32)
        self.mol_box = t(mol_box, np.int32)
        self.naf, self.nato = t(naf, np.int32), t(nato, np.int32)
        self.fclass = t(fclass, np.int32)
        self.xa, self.ya, self.za = t(xa, f32), t(ya, f32), t(za, f32)
        self.xadd, self.yadd, self.zadd = t(xadd, f32), t(yadd, f32), t(zadd, f32)
        self.tab, self.xstar, self.npairref = t(tabs, f32), t(xstars, f32), t(prs, np.int32)
        itype_all = np.concatenate(itype).astype(np.int32)
        pos = np.zeros((self.natom, 4), f32)
        naf_h, nato_h = np.concatenate(naf), np.concatenate(nato)
        xadd_h, yadd_h, zadd_h = np.concatenate(xadd), np.concatenate(yadd), np.concatenate(zadd)
        mol_of = np.repeat(np.arange(self.nmol), nato_h)
        pos[:, 0] = (np.concatenate(xa) + xadd_h[mol_of]).astype(f32)
        pos[:, 1] = (np.concatenate(ya) + yadd_h[mol_of]).astype(f32)
        pos[:, 2] = (np.concatenate(za) + zadd_h[mol_of]).astype(f32)
        pos[:, 3] = itype_all.view(f32)
        assert np.array_equal(naf_h, np.concatenate([[0], np.cumsum(nato_h)[:-1]]))
        self.pos = torch.from_numpy(pos.reshape(-1)).to(self.dev)
        z = lambda n, dt: torch.zeros(max(int(n), 1), dtype=dt, device=self.dev)  # noqa: E731
        self.cell_start = z(self.ncell + self.nbox, torch.int32)
        self.cell_mols = z(self.nmol, torch.int32)
        self.mol_cell = z(self.nmol + 2 * self.ncell + self.nbox, torch.int32)
        self.mol_cell[self.nmol + self.ncell + self.nbox:] = torch.from_numpy(np.concatenate(cell_box)).to(self.dev)
        self.slot_mol = z(self.nslot, torch.int32)
        self.slot_new = z(self.nslot * 64 * 4, torch.float32)
        self.slot_off = z(self.nslot * 64 * 4, torch.float32)
        self.slot_centre = z(self.nslot * 4, torch.float32)
        self.energy = z(self.nbox, torch.float64)
        self.emol = z(self.nmol, torch.float64)
        self.counters = z(self.nbox * 4, torch.int64)
        self.sweep_counter = z(1, torch.int64)
        self.status = z(1, torch.int32)
        c = Bmc()
        c.nbox, c.nmol, c.natom, c.ncell, c.nslot = self.nbox, self.nmol, self.natom, self.ncell, self.nslot
        c.threads = 256
        for k in ("slot_box", "mol_box", "naf", "nato", "fclass", "xa", "ya", "za", "xadd", "yadd", "zadd", "pos",
                  "tab", "xstar", "npairref", "cell_start", "cell_mols", "mol_cell", "slot_mol", "slot_new",
                  "slot_off", "slot_centre", "energy", "emol", "counters", "sweep_counter", "status"):
            setattr(c, k, _p(getattr(self, k)))
        c.box = _p(self.box_t)
        self.c = c
        # per-step buffers of the surrogate path
        self.rows = ((2 * self.nslot + 127) // 128) * 128
        self.x = self.y = self.resid = None
        self.graphs = {}

    # ------------------------------------------------------------------ calls
    def begin_sweep(self):
        check(self.lib.epsr_bmc_begin_sweep(C.byref(self.c), _stream()))

    def end_sweep(self):
        check(self.lib.epsr_bmc_end_sweep(C.byref(self.c), _stream()))

    def propose(self, step, x=None):
        check(self.lib.epsr_bmc_propose(C.byref(self.c), int(step), _p(x), _stream()))

    def decide(self, step, mode=0, y=None, target=None):
        check(self.lib.epsr_bmc_decide(C.byref(self.c), int(step), int(mode), _p(y), _p(target), _stream()))

    def total_energy(self):
        """Every box's total energy from scratch (bins the centres first)."""
        self.begin_sweep()
        check(self.lib.epsr_bmc_total_energy(C.byref(self.c), _stream()))
        return self.energy

    def feature_buffers(self):
        if self.x is None:
            self.x = torch.zeros(self.rows, FEAT_IN, dtype=torch.bfloat16, device=self.dev)
            self.y = torch.zeros(self.rows, dtype=torch.float32, device=self.dev)
            self.resid = torch.zeros(self.nslot, dtype=torch.float32, device=self.dev)
        return self.x, self.y

    def sweep(self, mode="plain", net=None, record=None):
        """One sweep of every box: mode "plain" (single-stage), "da" (delayed acceptance with the
        surrogate ``net``) or "record" (single-stage, features and beta*dE of every move appended
        to ``record``: a dict with "x" [rows][1280], "t" [pairs] tensors and "n" the pairs used)."""
        self.begin_sweep()
        T = self.steps_per_sweep
        for step in range(T):
            if mode == "plain":
                self.propose(step)
                self.decide(step, 0)
            elif mode == "da":
                x, y = self.feature_buffers()
                self.propose(step, x)
                net.forward(x, y)
                self.decide(step, 1, y, self.resid)
            elif mode == "record":
                n = record["n"]
                xs = record["x"][2 * n: 2 * (n + self.nslot)]
                ts = record["t"][n: n + self.nslot]
                self.propose(step, xs)
                self.decide(step, 2, None, ts)
                record["n"] = n + self.nslot
            else:
                raise ValueError(mode)
        self.end_sweep()

    def capture(self, mode="plain", net=None):
        """A CUDA graph of one sweep (replayed by run_graph); the sweep counter advances on the
        device, so every replay is a new sweep."""
        torch.cuda.synchronize()
        s = torch.cuda.Stream()
        s.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(s):
            self.sweep(mode, net)           # warm-up outside capture (lazy loading, workspaces)
        torch.cuda.current_stream().wait_stream(s)
        torch.cuda.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            self.sweep(mode, net)
        self.graphs[mode] = g
        return g

    def histograms(self, rminex=-2.0, tile=None):
        """Every box's partial g(r) histograms over all atom pairs in one launch (integer counts,
        normalised as atogen with every molecule an origin).  Returns per box (wav [2][npairs][ld],
        potex [npairs]) as device tensor views and the pair-updates counted."""
        tile = tile or getattr(self, "hist_tile", 1024)
        if getattr(self, "_hist", None) is None or self._hist.tile != tile:
            self._hist_setup(rminex, tile)
        check(self.lib.epsr_bmc_histograms(C.byref(self.c), C.byref(self._hist), self.h_counts.numel(), _stream()))
        out = []
        for b, s in enumerate(self.systems):
            ld = s.grid["npt"] + 1
            w0 = int(self._wav0[b])
            out.append((self.h_wav[w0:w0 + 2 * s.npairs * ld].view(2, s.npairs, ld),
                        self.h_potex[int(self._pair0[b]):int(self._pair0[b]) + s.npairs]))
        return out, self.h_pairs

    def _hist_setup(self, rminex, tile):
        items, hist0, wav0, npairs, npt1, ldw, pair0, type0 = [], [], [], [], [], [], [], []
        n1, n2, rmx, cfrac, csam = [], [], [], [], []
        h0 = w0 = p0 = t0 = 0
        max_bins = 1
        for b, s in enumerate(self.systems):
            ld = s.grid["npt"] + 1
            if s.npairs > 64:
                raise _lib.EpsrGpuError(4, "histograms: at most 64 pair types per box")
            for t_ in range(0, s.natom, tile):
                for o_ in range(0, s.natom, 256):
                    items.append((b, t_, o_))
            hist0.append(h0)
            wav0.append(w0)
            npairs.append(s.npairs)
            npt1.append(int(s.grid["npt1"]))
            ldw.append(ld)
            pair0.append(p0)
            type0.append(t0)
            n1.append(s.n1extr)
            n2.append(s.n2extr)
            rmx.append(np.full(s.npairs, rminex, f32))
            cfrac.append(s.cfrac.astype(f32))
            # atoms of every molecule by type (atogen's sampled-atom counts when all are sampled)
            cs = np.bincount(s.itype, minlength=s.ntype).astype(f32)
            csam.append(cs)
            max_bins = max(max_bins, s.npairs * ld + s.npairs)
            h0 += 2 * s.npairs * ld + s.npairs
            w0 += 2 * s.npairs * ld
            p0 += s.npairs
            t0 += s.ntype
        t = lambda a, dt: torch.from_numpy(np.ascontiguousarray(a, dtype=dt)).to(self.dev)  # noqa: E731
        self._h_items = t(np.array(items, np.int32).reshape(-1), np.int32)
        self._h_arrays = [t(hist0, np.int32), t(wav0, np.int32), t(npairs, np.int32), t(npt1, np.int32),
                          t(ldw, np.int32), t(pair0, np.int32), t(type0, np.int32), t(np.concatenate(n1), np.int32),
                          t(np.concatenate(n2), np.int32), t(np.repeat(np.arange(self.nmol),
                                                                     self.nato.cpu().numpy()), np.int32),
                          t(np.concatenate(rmx), f32), t(np.concatenate(cfrac), f32), t(np.concatenate(csam), f32)]
        self._wav0, self._pair0 = wav0, pair0
        self.h_counts = torch.zeros(max(h0, 1), dtype=torch.int64, device=self.dev)
        self.h_wav = torch.zeros(max(w0, 1), dtype=torch.float32, device=self.dev)
        self.h_potex = torch.zeros(max(p0, 1), dtype=torch.float32, device=self.dev)
        self.h_pairs = torch.zeros(self.nbox, dtype=torch.int64, device=self.dev)
        h = BmcHist()
        h.nitems, h.tile, h.max_bins = len(items), tile, max_bins
        h.items = _p(self._h_items)
        (h.hist0, h.wav0, h.npairs, h.npt1, h.ldw, h.pair0, h.type0, h.n1extr, h.n2extr, h.atom_mol, h.rminex,
         h.cfrac, h.csampled) = (_p(x) for x in self._h_arrays)
        h.counts, h.wav, h.potex, h.pairs = _p(self.h_counts), _p(self.h_wav), _p(self.h_potex), _p(self.h_pairs)
        self._hist = h

    def counters_host(self):
        return self.counters.cpu().numpy().reshape(self.nbox, 4)

    def check_status(self):
        v = int(self.status.item())
        if v:
            raise _lib.EpsrGpuError(5 if v == 1 else 3, "batched MC: " + {2: "partner list overflow"}.get(v, str(v)))

    def download(self):
        torch.cuda.synchronize()
        out = {k: getattr(self, k).cpu().numpy() for k in ("xa", "ya", "za", "xadd", "yadd", "zadd")}
        out["pos"] = self.pos.cpu().numpy().reshape(-1, 4)
        return out

    def box_slices(self, b):
        d = self.descs[b]
        return slice(d.mol0, d.mol0 + d.nmol), slice(d.atom0, d.atom0 + d.natom)
