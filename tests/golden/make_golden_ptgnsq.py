"""Golden vectors for the potential refinement of ptgnsq (epsr_standalone_rev3.py:3790-4021): the
per-data-set difference between the data and the weighted simulated S(Q), one fit_expansion per
data set on the reference's own Q-space basis (calc_pwrexpq), the coefficient increment
(:3948-3962) and generate_ep(.false.) (:4014), made by running the reference translation
(epsr26) on seeded state.

Run in a container where the reference is importable (it is read-only; nothing is written
there; ptgnsq's diagnostic file delfit.dat goes to a temporary folder that is removed):

    EPSR_REFERENCE=<reference checkout> PYTHONDONTWRITEBYTECODE=1 python tests/golden/make_golden_ptgnsq.py

The state: two data sets (no X-ray weighting, szeros 0, the whole Q range fitted), three atom
pairs in two coefficient sets (pairs 1 and 3 share set 1), real*8 weights cwt and cwtpot that
are not float32 values, seeded previous fit coefficients pcoefd, EP coefficients pcoefp and
tables.  tests/golden/ptgnsq.npz receives the inputs, the Q basis expsq the reference built,
the ran1 state before and after, and the refined state: pcoefd, pstepd, potnoi, pcoefp,
pwtold and the four EP tables.  tests/golden/ptgnsq_window.npz repeats it with the Q window
of :3856-3867 in use (qminp 1 A^-1, nqmin 6 and 4, the first data set extrapolated to
szeros = -0.3 below its window).  tests/golden/ptgnsq_xray.npz repeats the first with data set 1
an X-ray set (weights.xfile 1): its pairs are weighted by seeded Q-dependent real*8 weights
x_rayf0.weightx instead of cwt (:3849-3852); wq [set][pair][i] and the xray flags are saved.
"""

from __future__ import annotations

import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)
sys.path.insert(0, HERE)

from epsr_python_translation_b200 import configs  # noqa: E402
import refstate  # noqa: E402

f32 = np.float32
REF = refstate.reference_root()


def run(ep, out, nq=100, nterms=30, nits=200, seed=21, qminp=0.0, nqmin=(1, 1), szeros=(0.0, 0.0), xray=(0, 0)):
    from epsr26.common import clustercom, epsr16, epsrinput_par, molecom, potential_par as pp, weights, x_rayf0
    from epsr26.fortran import r4
    from epsr26.fortran.arrays import real_array
    from epsr26.library import auxiliary_routines
    rng = np.random.default_rng(seed)
    npairs, nsets, nfile = 3, 2, 2
    iref = [1, 2, 1]
    # r grid and EP tables (generate_ep's state)
    rmaxgr = 13.0
    g = configs.make_rgrid(0.03, rmaxgr, 9.0, 12.0)
    npt, npt2 = g["npt"], g["npt2"]
    dmax = f32(2.0 * rmaxgr)
    clustercom.dmax = dmax
    epsr16.npt, epsr16.npt2, epsr16.npt1 = npt, npt2, g["npt1"]
    epsr16.x[: npt + 1] = g["x"]
    epsr16.xstar[: npt + 1] = (g["x"] / dmax).astype(f32)
    epsr16.rho = f32(0.1)
    epsr16.cellst = f32(0.03)
    molecom.npairs = npairs
    molecom.simt = f32(0.008314) * f32(298.0)
    epsrinput_par.rminpt, epsrinput_par.rmaxpt, epsrinput_par.rbroad = f32(9.0), f32(12.0), f32(0.0)
    pp.pdstep = r4(0.1)
    pp.pdmin = r4(1.0) + pp.pdstep / epsrinput_par.rminpt
    pp.pdmax = epsrinput_par.rmaxpt
    pp.ncoeffp = nterms
    pp.psigma2 = r4(0.01)
    pp.gaussian = False
    pp.npairspcof = nsets
    for ip in range(1, npairs + 1):
        pp.irefpcof[ip] = iref[ip - 1]
    for k in range(1, nsets + 1):
        pp.npgauss[k] = 0
        pp.efacp[k] = f32(rng.uniform(0.5, 1.5))
    pc = np.zeros((nterms + 1, nsets), f32)
    pc[1] = 1.0
    pc[2:] = (rng.standard_normal((nterms - 1, nsets)) * 0.05).astype(f32)
    pp.pcoefp[1: nterms + 1, 1: nsets + 1] = pc[1:]
    wfac = configs.truncate_lj(g["x"].astype(np.float64), 9.0, 12.0).astype(f32)
    wfac[npt] = 0.0
    pp.wfac[: npt + 1] = wfac
    tabs = {}
    for k in ("ecoul", "xavs", "xavs1", "xavtot", "xavtot1"):
        v = (rng.standard_normal((npt + 1, npairs)) * 0.2).astype(f32)
        getattr(pp, k)[: npt + 1, 1: npairs + 1] = v
        tabs[k] = v
    pp.absolute_energy, pp.erequnit, pp.ereqstep = f32(3.0), f32(0.5), f32(0.0)
    pp.potfac, pp.potfacamp = f32(0.3), f32(0.5)
    pp.feedback = f32(1.0)
    pp.paccept = f32(0.05)
    pp.npits = pp.npitss = nits
    # data sets, weights and the previous fits
    q = configs.qgrid(nq, 0.3)
    epsr16.nfile = nfile
    epsr16.qminp, epsr16.qminm = f32(qminp), f32(0.0)
    cwt = rng.uniform(0.1, 0.6, (nfile, npairs))
    cwtpot = rng.uniform(0.1, 0.6, (npairs, nfile))
    pcoefd = np.zeros((nterms + 1, nfile), f32)
    pstepd = np.array([0.01, 0.02], f32)
    for d in range(1, nfile + 1):
        epsr16.nqmin[d], epsr16.nqmax[d] = int(nqmin[d - 1]), nq
        epsr16.sigma2[d] = pp.psigma2
        weights.xfile[d] = int(xray[d - 1])
        pp.npcoeff[d] = nterms
        pp.pstepd[d] = pstepd[d - 1]
        pcoefd[1:, d - 1] = (rng.standard_normal(nterms) * 0.01).astype(f32)
        pp.pcoefd[1: nterms + 1, d] = pcoefd[1:, d - 1]
        for ic in range(1, npairs + 1):
            weights.cwt[d, ic] = cwt[d - 1, ic - 1]
            weights.cwtpot[ic, d] = cwtpot[ic - 1, d - 1]
    qq = q.astype(np.float64)
    data = real_array(nq + 8, nfile)
    qwind = real_array(nq + 8, npairs)
    for d in range(1, nfile + 1):
        data[1: nq + 1, d] = (0.05 * np.sin(2.9 * qq[1:] + d) * np.exp(-0.05 * qq[1:])
                              + rng.normal(0, 0.005, nq)).astype(f32)
    for ic in range(1, npairs + 1):
        qwind[1: nq + 1, ic] = (0.04 * np.cos(2.1 * qq[1:] + ic) * np.exp(-0.04 * qq[1:])).astype(f32)
    wq = np.zeros((nfile, npairs, nq + 1))
    for d in range(1, nfile + 1):
        ix = int(xray[d - 1])
        if ix > 0:
            w = rng.uniform(0.05, 0.5, (npairs, nq)) * np.exp(-0.01 * qq[1:])
            x_rayf0.weightx[1: nq + 1, 1: npairs + 1, ix] = w.T
            wq[d - 1, :, 1:] = w
    out["wq"], out["xray"] = wq, np.array(xray, np.int32)
    qa = real_array(nq + 8)
    qa[1: nq + 1] = q[1:]
    for _ in range(53):
        auxiliary_routines.ran1()
    out.update({"q": q, "data": np.array(data[: nq + 1, 1: nfile + 1]).T.copy(),
                "qwind": np.array(qwind[: nq + 1, 1: npairs + 1]).T.copy(), "cwt": cwt, "cwtpot": cwtpot.T.copy(),
                "efacp": np.array(pp.efacp[1: nsets + 1], f32), "iref": np.array(iref, np.int32) - 1,
                "pcoefd_in": pcoefd.T.copy(), "pstepd_in": pstepd, "pcoefp_in": pc.T.copy(), "wfac": wfac,
                "x": g["x"], "xstar": (g["x"] / dmax).astype(f32),
                "dims": np.array([npairs, nsets, nfile, nq, nterms, nits, npt, npt2]),
                "scal": np.array([dmax, 3.0, 0.5, 0.0, 0.5, 0.3, 0.01], f32),
                "basis": np.array([pp.pdmin, pp.pdstep, pp.pdmax, pp.psigma2, epsr16.rho], f32)})
    for k, v in tabs.items():
        out["in_" + k] = v.T.copy()
    for k, v in refstate.ran1_state().items():
        out["ran1_before_" + k] = v
    szeros_a = real_array(8)
    szeros_a[1: nfile + 1] = np.array(szeros, f32)
    out["window"] = np.array([qminp, *nqmin, *szeros], f32)
    rminp = real_array(8)
    potnoi = real_array(8)
    cwd = os.getcwd()
    with tempfile.TemporaryDirectory(dir=HERE) as tmp:
        os.chdir(tmp)
        try:
            ep.ptgnsq(1, nq, qa, real_array(2, 8, 8), data, qwind, f32(9.0), f32(12.0), szeros_a, real_array(8),
                      real_array(8), rminp, potnoi, f32(0.1), f32(0.0), f32(0.0), 0)
        finally:
            os.chdir(cwd)
    out["expsq"] = np.array(pp.expsq[1: nq * nterms + 1], f32)
    out["pcoefd"] = np.array(pp.pcoefd[: nterms + 1, 1: nfile + 1], f32).T.copy()
    out["pstepd"] = np.array(pp.pstepd[1: nfile + 1], f32)
    out["potnoi"] = np.array(potnoi[1: nfile + 1], f32)
    out["pcoefp"] = np.array(pp.pcoefp[: nterms + 1, 1: nsets + 1], f32).T.copy()
    out["pwtold"] = np.array(pp.pwtold[: nterms + 1], f32)
    for k in ("xavs", "xavs1", "xavtot", "xavtot1"):
        out[k] = np.array(getattr(pp, k)[: npt + 1, 1: npairs + 1], f32).T.copy()
    for k, v in refstate.ran1_state().items():
        out["ran1_after_" + k] = v


if __name__ == "__main__":
    common, _ = refstate.load_reference(os.path.join(REF, "src"))
    import importlib
    ep = importlib.import_module("epsr26.programs.epsr_standalone_rev3")
    for name, kw in (("ptgnsq", {}),
                     # the Q window: data from Q index 6 (set 1) and 4 (set 2), Q below 1.0 A^-1 outside it,
                     # set 1 extrapolated to szeros at Q = q(1)
                     ("ptgnsq_window", dict(qminp=1.0, nqmin=(6, 4), szeros=(-0.3, 0.0))),
                     # data set 1 an X-ray set with Q-dependent pair weights
                     ("ptgnsq_xray", dict(xray=(1, 0)))):
        out = {}
        common.reset()
        run(ep, out, **kw)
        path = os.path.join(HERE, name + ".npz")
        np.savez_compressed(path, **out)
        print("wrote", path, "mcall", int(out["ran1_after_mcall"]) - int(out["ran1_before_mcall"]))
