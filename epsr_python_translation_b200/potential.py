"""The empirical potential (EP) rebuilt from its coefficients: generate_ep
(epsr_standalone_rev3.py:5876-6022) on the device, with the basis matrix built once on the
host (calc_pwrexpr_grad :5230 or calc_gaussr_grad :5046, the C library's logf/expf as the
reference).

Layouts (the device form of the reference's 1-based COMMON arrays of potential_par):
coefficient sets ``pcoefp`` (nsets, ldc) with coefficient ic of set k at [k, ic]; tables
``xavs``, ``xavs1``, ``xavtot``, ``xavtot1``, ``ecoul`` (npairs, ld) with the r index j at
[pair, j]; ``xstar`` and ``wfac`` (ld,); ``iref`` the 0-based set of each pair (irefpcof - 1).
"""

from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib
from ._lib import check

f32 = np.float32
TABLES = ("xavs", "xavs1", "xavtot", "xavtot1")


def _p(t):
    return C.c_void_p(t.data_ptr())


def _s():
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def basis(npt2, nterms, x, gaussian, pdmin, pdstep, pdmax, psigma2, rho, rbroad, rmin=0.0, fbroad=1.0, ncfirst=0):
    """The r-space basis generate_ep builds on entry (epsr_standalone_rev3.py:5907-5912):
    calc_gaussr_grad when ``gaussian`` else calc_pwrexpr_grad, on points x[1..npt2] (x 1-based).
    Host computation.  Returns (expgr (npt2*nterms,) float32 -- the reference's
    expgr(1..npt2*nterms) --, ncfirst)."""
    lib = _lib.load()
    xs = np.ascontiguousarray(np.asarray(x, f32)[: npt2 + 1])
    out = np.zeros(int(npt2) * int(nterms), f32)
    nc = C.c_int32(int(ncfirst))
    xp, op = xs.ctypes.data_as(C.c_void_p), out.ctypes.data_as(C.c_void_p)
    if gaussian:
        rc = lib.epsr_calc_gaussr_grad(int(npt2), int(nterms), f32(pdstep), f32(pdmax), f32(psigma2), f32(rho), xp,
                                       op, f32(rmin), C.byref(nc), f32(fbroad), f32(rbroad))
    else:
        rc = lib.epsr_calc_pwrexpr_grad(int(npt2), int(nterms), f32(pdmin), f32(pdstep), f32(pdmax), f32(psigma2),
                                        f32(rho), xp, op, f32(rmin), C.byref(nc), f32(fbroad), f32(rbroad))
    check(rc)
    return out, int(nc.value)


def generate_ep(npt, npt2, nterms, expgr, pcoefp, iref, dmax, xstar, wfac, ecoul, tabs, pwtold, absolute_energy,
                erequnit, ereqstep, potfacamp, potfac, changepotfac=True, result=None):
    """generate_ep epsr_standalone_rev3.py:5876-6022 on device tensors, in place: ``tabs``
    (dict of the four tables), ``pcoefp``, ``pwtold`` (nterms+1,) and ``potfac`` (1,).
    ``iref`` is a host int array.  Returns the device tensor (energabs, pressfac)."""
    lib = _lib.load(require_device=True)
    npairs, ld = ecoul.shape
    nsets, ldc = pcoefp.shape
    if result is None:
        result = torch.zeros(2, dtype=torch.float32, device=ecoul.device)
    ir = np.ascontiguousarray(np.asarray(iref, np.int32))
    if ir.shape[0] != npairs:
        raise ValueError(f"iref has {ir.shape[0]} entries for {npairs} pairs")
    for t in (expgr, pcoefp, xstar, wfac, ecoul, pwtold, potfac, result, *tabs.values()):
        if t.dtype != torch.float32 or not t.is_contiguous() or not t.is_cuda:
            raise ValueError("generate_ep takes contiguous float32 device tensors")
    if pwtold.numel() < nterms + 1 or potfac.numel() < 1 or result.numel() < 2 or xstar.numel() < ld or \
            wfac.numel() < ld or expgr.numel() < npt2 * nterms:
        raise ValueError("generate_ep: pwtold, potfac, result, xstar, wfac or expgr is too short")
    for k in TABLES:
        if tuple(tabs[k].shape) != (npairs, ld):
            raise ValueError(f"table {k} has shape {tuple(tabs[k].shape)}, not {(npairs, ld)}")
    check(lib.epsr_generate_ep(int(npairs), int(npt), int(npt2), int(nterms), _p(expgr), _p(pcoefp), int(nsets),
                               int(ldc), ir.ctypes.data_as(C.c_void_p), f32(dmax), _p(xstar), _p(wfac), _p(ecoul),
                               _p(tabs["xavs"]), _p(tabs["xavs1"]), _p(tabs["xavtot"]), _p(tabs["xavtot1"]), int(ld),
                               _p(pwtold), f32(absolute_energy), f32(erequnit), f32(ereqstep), f32(potfacamp),
                               _p(potfac), int(bool(changepotfac)), _p(result), _s()))
    return result


def ep_update(pcoefp, iref, efacp, cwtpot, pwtold, pfact):
    """ptgnsq's coefficient increment (epsr_standalone_rev3.py:3948-3962) after the fits of all
    data sets, in place on ``pcoefp`` (nsets, ldc): efacp (nsets,), cwtpot (ndata, npairs,
    float64: real*8 in the reference) and pwtold (ndata, ldw) device tensors, iref a host int
    array, pfact the potential factor."""
    if cwtpot.dtype != torch.float64:
        raise ValueError("ep_update: cwtpot is real*8 in the reference; pass a float64 tensor")
    lib = _lib.load(require_device=True)
    nsets, ldc = pcoefp.shape
    ndata, npairs = cwtpot.shape
    ldw = pwtold.shape[1]
    ir = np.ascontiguousarray(np.asarray(iref, np.int32))
    if ir.shape[0] != npairs or pwtold.shape[0] != ndata or efacp.numel() < nsets:
        raise ValueError("ep_update: inconsistent shapes")
    check(lib.epsr_ep_update(int(ndata), int(npairs), int(ldw - 1), _p(pcoefp), int(nsets), int(ldc),
                             ir.ctypes.data_as(C.c_void_p), _p(efacp), _p(cwtpot), _p(pwtold), int(ldw), f32(pfact),
                             _s()))


def pack_tables(xavs, xavs1, ecoul, ecoul1, tab):
    """The packed {xavs, xavs1, ecoul, ecoul1} table of the energy kernels (npairs*ld*4,)."""
    lib = _lib.load(require_device=True)
    npairs, ld = xavs.shape
    if tab.numel() < 4 * npairs * ld or any(tuple(t.shape) != (npairs, ld) for t in (xavs1, ecoul, ecoul1)):
        raise ValueError("pack_tables: inconsistent shapes")
    check(lib.epsr_pack_tables(int(npairs), int(ld), _p(xavs), _p(xavs1), _p(ecoul), _p(ecoul1), _p(tab), _s()))


RP_TABLES = ("epot", "epot1", "ecoul", "ecoul1", "xav", "xav1")


def reference_potential(x, xstar, wfac, wfacc, npt, npt2, n1extr, n2extr, irefpcof, qradius, ecor, qcor, dcor, coulfac,
                        pcoefex, rminex, power, ecore, dcore, sizefactor=1.0, refpotfac=1.0, expecf=0.0,
                        expecfpwr=0.0, harmonic=False, modmorse=False, coul_intra=False, coul_intra_fac=0.0,
                        npgauss=None, wpgauss=None, rpgauss=None, hpgauss=None, out=None):
    """generate_mp + generate_rp (ato_manipulation_rev4.py:2816, epsr_standalone_rev3.py:5675) on
    the host through the library: returns the tables epot, epot1, ecoul, ecoul1, xav, xav1
    ((npairs, npt+1) float32 each, r index 1-based).  Types and sets are 0-based; the Gaussian
    arrays are (nsets, maxgauss)."""
    lib = _lib.load()
    npairs = len(n1extr)
    ld = int(npt) + 1
    a = lambda v, dt=f32: np.ascontiguousarray(np.asarray(v, dt))  # noqa: E731
    nsets = len(coulfac)
    npg = a(np.zeros(nsets) if npgauss is None else npgauss, np.int32)
    maxg = 0 if wpgauss is None else np.asarray(wpgauss).reshape(nsets, -1).shape[1]
    keep = dict(x=a(x)[:ld], xstar=a(xstar)[:ld], wfac=a(wfac)[:ld], wfacc=a(wfacc)[:ld], n1extr=a(n1extr, np.int32),
                n2extr=a(n2extr, np.int32), irefpcof=a(irefpcof, np.int32), qradius=a(qradius), ecor=a(ecor),
                qcor=a(qcor), dcor=a(dcor), coulfac=a(coulfac), pcoefex=a(pcoefex), rminex=a(rminex), npgauss=npg)
    for k, v in (("wpgauss", wpgauss), ("rpgauss", rpgauss), ("hpgauss", hpgauss)):
        keep[k] = a(np.zeros((nsets, 1)) if v is None else np.asarray(v).reshape(nsets, -1))
    out = out if out is not None else {k: np.zeros((npairs, ld), f32) for k in RP_TABLES}
    r = _lib.Rp()
    r.npairs, r.npt, r.npt2, r.ld = npairs, int(npt), int(npt2), ld
    for k, v in keep.items():
        setattr(r, k, v.ctypes.data_as(C.c_void_p))
    for k in RP_TABLES:
        if out[k].shape != (npairs, ld) or out[k].dtype != f32 or not out[k].flags.c_contiguous:
            raise ValueError(f"reference_potential: table {k} must be a contiguous float32 ({npairs}, {ld}) array")
        setattr(r, k, out[k].ctypes.data_as(C.c_void_p))
    r.power, r.ecore, r.dcore, r.sizefactor = (float(f32(v)) for v in (power, ecore, dcore, sizefactor))
    r.refpotfac, r.expecf, r.expecfpwr = (float(f32(v)) for v in (refpotfac, expecf, expecfpwr))
    r.harmonic, r.modmorse, r.coul_intra = int(bool(harmonic)), int(bool(modmorse)), int(bool(coul_intra))
    r.coul_intra_fac = float(f32(coul_intra_fac))
    r.maxgauss = int(maxg)
    check(lib.epsr_generate_rp(C.byref(r)))
    return out
