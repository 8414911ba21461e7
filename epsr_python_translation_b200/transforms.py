"""Device calls for gensq, stog and fit_expansion on PyTorch tensors (C ABI wrappers)."""

from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib
from ._lib import check

f32 = np.float32


def _p(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


def _s():
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def _dev(a, dtype=torch.float32):
    if isinstance(a, torch.Tensor):
        return a.to(device="cuda", dtype=dtype).contiguous()
    return torch.from_numpy(np.ascontiguousarray(a)).to(device="cuda", dtype=dtype)


def gensq(nq, npt1, wav, ldw, foqols, sj, si, ycoh, n2extr, natomsphere, npairs):
    """gensq epsr_standalone_rev3.py:4731.  wav (device, 2*npairs*ldw); foqols with strides
    (sj, si) for (r index, Q index).  Returns sofq (device, 2*npairs*(nq+1))."""
    lib = _lib.load(require_device=True)
    out = torch.zeros(2 * npairs * (nq + 1), dtype=torch.float32, device="cuda")
    fq = _dev(foqols)
    yc = _dev(ycoh)
    n2 = _dev(n2extr, torch.int32)
    ns = _dev(natomsphere)
    check(lib.epsr_gensq(nq, npairs, npt1, _p(wav), ldw, _p(fq), sj, si, _p(yc), _p(n2), _p(ns), _p(out), _s()))
    return out


def ptgnsq_difference(data, cwt, qwind, out=None, q=None, nqmin=None, nqmax=None, szeros=None, qmin=0.0, wq=None,
                      xray=None):
    """The simulated fit of each data set and its negated difference from the data
    (ptgnsq epsr_standalone_rev3.py:3844-3867): -(data - cwt @ qwind), the sum over atom
    pairs sequential, each step in double and rounded to float32 (the weights are real*8).
    data (ndata, nq+1) float32, cwt (ndata, npairs) float64, qwind (npairs, nq+1) float32,
    all on the device.  With q ((nq+1,), 1-based) the reference's Q window applies: per data
    set nqmin, nqmax, szeros (host or device; None: 1, nq, 0) and qmin (qminp, or qminm when
    qminp <= 0).  X-ray data sets: xray (ndata,) flags and wq (ndata, npairs, nq+1) float64
    Q-dependent weights used in place of cwt where the flag is set."""
    if cwt.dtype != torch.float64:
        raise ValueError("ptgnsq_difference: cwt is real*8 in the reference; pass a float64 tensor")
    lib = _lib.load(require_device=True)
    ndata, ld = data.shape
    npairs = cwt.shape[1]
    if out is None:
        out = torch.empty_like(data)
    win = []
    if q is not None:
        win = [_dev(q), None if nqmin is None else _dev(nqmin, torch.int32),
               None if nqmax is None else _dev(nqmax, torch.int32), None if szeros is None else _dev(szeros)]
    qp, n0, n1, sz = (win + [None] * 4)[:4]
    wqd = None if wq is None else _dev(wq, torch.float64)
    if wqd is not None and tuple(wqd.shape) != (ndata, npairs, ld):
        raise ValueError(f"ptgnsq_difference: wq must be (ndata, npairs, nq+1) = {(ndata, npairs, ld)}")
    xrd = None if xray is None else _dev(xray, torch.int32)
    check(lib.epsr_ptgnsq_difference(ndata, npairs, ld - 1, _p(data), _p(cwt), _p(qwind), _p(qp), _p(n0), _p(n1), _p(sz),
                                     f32(qmin), _p(wqd), _p(xrd), _p(out), _s()))
    return out


GR_ARRAYS = ("gorintra", "gorinter", "gr2intra", "gr2inter", "entsig")
SQ_ARRAYS = ("soqintra", "soqinter", "sq2intra", "sq2inter")


def sumgr(nz, wav, ycoh, fc1, fc2, acc):
    """sumgr epsr_standalone_rev3.py:3578-3637 on the device: folds the new partial g(r) into
    the running means and error bars with weights fc2 (old) and fc1 (new) and recomputes the
    zero limit.  wav (device, 2*npairs*ldw); ycoh (device, ldw); acc a dict of device
    float32 tensors (npairs, ldw) named as GR_ARRAYS, updated in place."""
    lib = _lib.load(require_device=True)
    npairs, ldw = acc["gorintra"].shape
    check(lib.epsr_sumgr(int(nz), npairs, _p(wav), ldw, _p(ycoh), float(fc1), float(fc2),
                         *(_p(acc[k]) for k in GR_ARRAYS), _s()))
    return acc


def sumsq(nq, qwind, fc1, fc2, acc):
    """sumsq epsr_standalone_rev3.py:3642-3677 on the device: the same for the partial S(Q).
    qwind (device, 2*npairs*ldq), gensq's output; acc a dict of device float32 tensors
    (npairs, ldq) named as SQ_ARRAYS, updated in place."""
    lib = _lib.load(require_device=True)
    npairs, ldq = acc["soqintra"].shape
    check(lib.epsr_sumsq(int(nq), npairs, _p(qwind), ldq, float(fc1), float(fc2),
                         *(_p(acc[k]) for k in SQ_ARRAYS), _s()))
    return acc


def stog(rho, q, sofq_pairs, r, nqmin, nqmax, xwt):
    """stog ato_manipulation_rev4.py:4067.  q (ldq,), sofq_pairs (npairs, ldq), r (nr+1,)."""
    lib = _lib.load(require_device=True)
    npairs, ldq = sofq_pairs.shape
    nr = r.shape[0] - 1
    qd, sd, rd, xd = _dev(q), _dev(sofq_pairs), _dev(r), _dev(xwt)
    lo, hi = _dev(nqmin, torch.int32), _dev(nqmax, torch.int32)
    out = torch.zeros(npairs * (nr + 1), dtype=torch.float32, device="cuda")
    nb = int(lib.epsr_stog_scratch_bytes(npairs, ldq))
    scr = torch.empty(nb, dtype=torch.uint8, device="cuda")
    check(lib.epsr_stog(float(f32(rho)), _p(qd), ldq, _p(sd), _p(rd), nr, npairs, _p(lo), _p(hi), _p(xd), _p(out),
                        _p(scr), nb, _s()))
    return out.view(npairs, nr + 1)


def fit_expansion(yin, expr, wtold, stepr, nmin, npt, ncfirst, nterms, nits, nfreq, ran1_t, acceptr=0.0,
                  rejrat=0.0, chisqnew=0.0, strict=True):
    """fit_expansion epsr_standalone_rev3.py:4806 (1-based arrays).  ran1_t: device int32[35]."""
    lib = _lib.load(require_device=True)
    y = _dev(yin)
    e = _dev(expr)
    wt = torch.zeros(nterms + 1, dtype=torch.float32, device="cuda")
    wto = _dev(wtold).clone()
    yout = torch.zeros(npt + 1, dtype=torch.float32, device="cuda")
    scal = np.array([stepr, acceptr, rejrat, chisqnew], f32)
    nb = lib.epsr_fit_expansion_scratch_bytes(npt, nterms)
    scr = torch.empty(int(nb), dtype=torch.uint8, device="cuda")
    trials = np.zeros(1, np.int64)
    check(lib.epsr_fit_expansion(_p(y), _p(e), _p(yout), _p(wt), _p(wto), scal.ctypes.data_as(C.c_void_p), nmin, npt,
                                 ncfirst, nterms, nits, nfreq, _p(ran1_t), _p(scr), scr.numel(), 1 if strict else 0,
                                 trials.ctypes.data_as(C.c_void_p), _s()))
    return dict(wt=wt, wtold=wto, yout=yout, stepr=f32(scal[0]), acceptr=f32(scal[1]), rejrat=f32(scal[2]),
                chisq=f32(scal[3]), trials=int(trials[0]))


def fit_expansion_batch(yin, expr, wtold, stepr, nmin, npt, ncfirst, nterms, nits, nfreq, ran1_t, strict=True,
                        scratch=None):
    """fit_expansion for each row of yin (nprob, npt+1) in turn on one ran1 stream, in one
    launch (the reference's successive calls per data set, epsr_standalone_rev3.py:3936).
    wtold (nprob, nterms+1) and stepr (nprob,) are the per-set inputs.  Returns a dict of
    per-set outputs (tensors with a leading nprob axis, host arrays for the scalars)."""
    lib = _lib.load(require_device=True)
    y = _dev(yin)
    nprob = y.shape[0]
    e = _dev(expr)
    wt = torch.zeros(nprob, nterms + 1, dtype=torch.float32, device="cuda")
    wto = _dev(wtold).clone()
    yout = torch.zeros(nprob, npt + 1, dtype=torch.float32, device="cuda")
    scal = np.zeros((nprob, 4), f32)
    scal[:, 0] = np.asarray(stepr, f32)
    nb = int(lib.epsr_fit_expansion_batch_scratch_bytes(nprob, npt, nterms))
    scr = scratch if scratch is not None and scratch.numel() >= nb else torch.empty(nb, dtype=torch.uint8,
                                                                                     device="cuda")
    trials = np.zeros(nprob, np.int64)
    check(lib.epsr_fit_expansion_batch(nprob, _p(y), _p(e), _p(yout), _p(wt), _p(wto),
                                       scal.ctypes.data_as(C.c_void_p), nmin, npt, ncfirst, nterms, nits, nfreq,
                                       _p(ran1_t), _p(scr), scr.numel(), 1 if strict else 0,
                                       trials.ctypes.data_as(C.c_void_p), _s()))
    return dict(wt=wt, wtold=wto, yout=yout, stepr=scal[:, 0].copy(), acceptr=scal[:, 1].copy(),
                rejrat=scal[:, 2].copy(), chisq=scal[:, 3].copy(), trials=trials)
