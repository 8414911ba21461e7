"""ctypes binding of libepsr_gpu.so (the C ABI declared in include/epsr_gpu.h).

The device library is the only compute path: if it is missing or no sm_100 device is
visible, calls raise ``EpsrGpuError`` -- there is no CPU fallback.
"""

from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIBPATH = os.path.join(HERE, "libepsr_gpu.so")

P = C.c_void_p
I32 = C.c_int32
I64 = C.c_int64
F32 = C.c_float


class EpsrGpuError(RuntimeError):
    """A nonzero status from the C ABI (code, message)."""

    def __init__(self, code, msg):
        super().__init__(f"epsr_gpu error {code}: {msg}")
        self.code = code


class Box(C.Structure):
    _fields_ = [("nmol", I32), ("natom", I32), ("ntype", I32), ("npairs", I32), ("nmoltype", I32),
                ("naf", P), ("nato", P), ("mtype", P), ("itype", P), ("xa", P), ("ya", P), ("za", P),
                ("xadd", P), ("yadd", P), ("zadd", P), ("pos", P), ("npairref", P), ("xstar", P), ("tab", P),
                ("ld", I32), ("npt2", I32), ("izcut", I32), ("stepcl", F32), ("cubic", I32), ("lat", F32 * 6),
                ("maxat", I32)]


class Cells(C.Structure):
    _fields_ = [("ncelldiva", I32), ("ncelldivb", I32), ("ncelldivc", I32), ("ncell", I32), ("ncellneighb", I32),
                ("maxcellno", I32), ("molcellno", P), ("cell_start", P), ("cell_mols", P), ("offsets", P),
                ("nnbrefmax", I32)]


class Store(C.Structure):
    _fields_ = [("nnbrefmax", I32), ("capacity", I32), ("nergpairm", P), ("molergpair", P), ("ergpairref", P),
                ("ergpair", P), ("nergpair", P), ("mirror", P)]


class Mc(C.Structure):
    _fields_ = [("simt", F32), ("rejrate", F32), ("stepr", F32), ("stepm", F32), ("trstepmax", F32),
                ("trstepmin", F32), ("ireset", I32), ("wholerot", P), ("wholetrans", P), ("internrot", P),
                ("interntrans", P), ("nwhole", P), ("nmovem", P), ("nstepreject", P), ("fadds", P), ("ran1", P),
                ("cos_override", P), ("trace_den", P), ("trace_acc", P), ("strict", I32),
                ("status", P), ("intra", P), ("rot_nrf", P), ("rot_nrl", P), ("rot_axis", P), ("rot_first", P),
                ("rot_last", P), ("rot_atoms", P), ("stepri", F32), ("rotcycle", I32), ("ninter", P),
                ("faddbs", P), ("ahead", P), ("ahead_cap", I64)]


class Mlp(C.Structure):
    """epsr_mlp_t: the surrogate network's parameters, gradients and Adam moments (device)."""
    _fields_ = [("w1", P), ("b1", P), ("w2", P), ("b2", P), ("w3", P), ("b3", P), ("w1h", P), ("w2h", P),
                ("w2th", P), ("dw1", P), ("db1", P), ("dw2", P), ("db2", P), ("dw3", P), ("db3", P), ("m1", P),
                ("v1", P), ("status", P)]


class Intra(C.Structure):
    """epsr_intra_t: the intramolecular model of en_atom_intra (device pointers)."""
    _fields_ = [("nbond", P), ("iabond", P), ("tbond", P), ("maxbond", I32), ("imageatom", P), ("qtype", P),
                ("amassa", P), ("amassr", P), ("xav", P), ("xav1", P), ("ngrot", P), ("stepcl", F32),
                ("sizefactor", F32), ("tempb", F32), ("tempang", F32), ("simt", F32), ("refine_intra", I32),
                ("refine_intra_fac", F32), ("ndih", I32), ("grp_nrf", P), ("grp_nrl", P), ("grp_axis", P),
                ("grp_dih0", P), ("grp_isdih", P), ("dih_atoms", P), ("dih_cos", P), ("dih_sin", P),
                ("tempdih", F32)]


class Rp(C.Structure):
    """epsr_rp_t: inputs and outputs of generate_mp + generate_rp (host pointers)."""
    _fields_ = [("npairs", I32), ("npt", I32), ("npt2", I32), ("ld", I32), ("x", P), ("xstar", P), ("wfac", P),
                ("wfacc", P), ("power", F32), ("ecore", F32), ("dcore", F32), ("sizefactor", F32),
                ("refpotfac", F32), ("expecf", F32), ("expecfpwr", F32), ("harmonic", I32), ("modmorse", I32),
                ("coul_intra", I32), ("coul_intra_fac", F32), ("n1extr", P), ("n2extr", P), ("irefpcof", P),
                ("qradius", P), ("ecor", P), ("qcor", P), ("dcor", P), ("coulfac", P), ("pcoefex", P),
                ("rminex", P), ("npgauss", P), ("maxgauss", I32), ("wpgauss", P), ("rpgauss", P), ("hpgauss", P),
                ("epot", P), ("epot1", P), ("ecoul", P), ("ecoul1", P), ("xav", P), ("xav1", P)]


class Iteration(C.Structure):
    """epsr_iteration_t: one EPSR iteration of the path, driven natively."""
    _fields_ = [("box", P), ("mc", P),
                ("nmolcell", I32), ("rmax", F32), ("lat6", F32 * 6), ("lat9", F32 * 9),
                ("cell_molcellno", P), ("cell_start", P), ("cell_mols", P), ("cell_offsets", P),
                ("cell_scratch", P), ("cell_scratch_n", I64),
                ("store_m", I32), ("store_capacity", I32),
                ("nergpairm", P), ("molergpair", P), ("ergpairref", P), ("mirror", P), ("nergpair", P),
                ("ergpair", P), ("eintra", P), ("ntimes", I32),
                ("npt1", I32), ("natomr", I32), ("ngrsamples", I32), ("sizefactor", F32), ("dmax", F32),
                ("rminex", P), ("cfrac", P), ("ycoh", P), ("n1extr", P), ("n2extr", P),
                ("wav", P), ("ldw", I32), ("potex", P), ("counts", P),
                ("nq", I32), ("ndata", I32), ("foqols", P), ("foqols_sj", I64), ("foqols_si", I64),
                ("natomsphere", P), ("sofq", P), ("data", P), ("cwt", P), ("dt", P),
                ("expr", P), ("nterms", I32), ("ncfirst", I32), ("nits", I32), ("nfreq", I32),
                ("fit_wt", P), ("fit_wtold", P), ("fit_yout", P), ("fit_scal_host", P), ("fit_trials_host", P),
                ("rho", F32), ("q", P), ("r", P), ("nr", I32), ("nqmin", P), ("nqmax", P), ("xwt", P),
                ("gofr", P), ("nsum", I32), ("soqintra", P), ("soqinter", P), ("sq2intra", P), ("sq2inter", P),
                ("gorintra", P), ("gorinter", P), ("gr2intra", P), ("gr2inter", P), ("entsig", P),
                ("refine", I32), ("pcoefp", P), ("nsets", I32), ("ldc", I32), ("irefpcof_host", P), ("efacp", P),
                ("cwtpot", P), ("expgr", P), ("wfac", P), ("ecoul", P), ("ecoul1", P), ("xavs", P), ("xavs1", P),
                ("xavtot", P), ("xavtot1", P), ("ep_pwtold", P), ("potfac", P), ("ep_result", P), ("pfact", F32),
                ("absolute_energy", F32), ("erequnit", F32), ("ereqstep", F32), ("potfacamp", F32), ("tab", P),
                ("intra", I32), ("nisum", I32), ("stepmi", F32), ("intra_model", P), ("faddbs", P),
                ("eintra_work", P), ("nmovei", P),
                ("scratch", P), ("scratch_bytes", I64), ("strict", I32), ("stage_events", P * 20),
                ("rotfreq", I32)]


class IterationReport(C.Structure):
    _fields_ = [("nnbrefmax", I32), ("ftest", F32 * 2), ("ngrsamples", I32), ("pair_updates", I64),
                ("press", C.c_double * 2), ("nisum", I32)]


_SIGS = {
    "epsr_last_error": (C.c_char_p, []),
    "epsr_version": (C.c_char_p, []),
    "epsr_device_count": (C.c_int, []),
    "epsr_ran1_fill": (C.c_int, [P, P, I64, P]),
    "epsr_cell_dims": (C.c_int, [I32, I32, P, P]),
    "epsr_cell_list": (C.c_int, [P, P, P, I32, I32, F32, P, P, C.POINTER(Cells), P, I64, P]),
    "epsr_nnbrefmax": (C.c_int, [C.POINTER(Cells), P, P, P]),
    "epsr_box_positions": (C.c_int, [C.POINTER(Box), P]),
    "epsr_fmolec1_scratch_bytes": (I64, [I32, I32, I32]),
    "epsr_fmolec1": (C.c_int, [C.POINTER(Box), C.POINTER(Cells), P, C.POINTER(Store), P, I64, I32, P, P]),
    "epsr_molfit_scratch_bytes": (I64, [I32, I32, I32]),
    "epsr_molfit_spec_scratch_bytes": (I64, [I32, I32, I32, I32]),
    "epsr_molfit": (C.c_int, [C.POINTER(Box), C.POINTER(Cells), C.POINTER(Store), C.POINTER(Mc), P, I64, P]),
    "epsr_en_change": (C.c_int, [C.POINTER(Box), C.POINTER(Store), I32, P, P, P]),
    "epsr_en_mole_pair": (C.c_int, [C.POINTER(Box), P, P, I32, P, P]),
    "epsr_atogen": (C.c_int, [C.POINTER(Box), I32, F32, F32, P, P, P, P, P, I32, P, P, P, I32, P, P, P, I64, P]),
    "epsr_atogen_scratch_bytes": (I64, [I32, I32, I32, I32]),
    "epsr_atogen_last_pair_updates": (I64, []),
    "epsr_atogen_noalloc": (C.c_int, [C.POINTER(Box), I32, F32, F32, P, P, P, P, P, I32, P, P, P, I32, P, P]),
    "epsr_timing_enable": (C.c_int, [I32]),
    "epsr_umma_gemm_f32": (C.c_int, [P, I32, P, I32, I32, I32, P, I32, I32, P, P]),
    "epsr_bmc_begin_sweep": (C.c_int, [P, P]),
    "epsr_bmc_propose": (C.c_int, [P, I32, P, P]),
    "epsr_bmc_decide": (C.c_int, [P, I32, I32, P, P, P]),
    "epsr_bmc_end_sweep": (C.c_int, [P, P]),
    "epsr_bmc_total_energy": (C.c_int, [P, P]),
    "epsr_bmc_histograms": (C.c_int, [P, P, I64, P]),
    "epsr_mlp_work_bytes": (I64, [I32]),
    "epsr_mlp_sync_weights": (C.c_int, [C.POINTER(Mlp), P]),
    "epsr_mlp_forward": (C.c_int, [C.POINTER(Mlp), P, I32, P, P, I64, P]),
    "epsr_mlp_train_step": (C.c_int, [C.POINTER(Mlp), P, P, I64, I32, I32, P, F32, I32, P, P, I64, P]),
    "epsr_timing_read": (C.c_int, [C.c_char_p, P, P]),
    "epsr_press": (C.c_int, [C.POINTER(Box), C.POINTER(Store), I32, P, I64, I32, P, P]),
    "epsr_press_scratch_bytes": (I64, [I32, I32]),
    "epsr_gensq": (C.c_int, [I32, I32, I32, P, I32, P, I64, I64, P, P, P, P, P]),
    "epsr_ptgnsq_difference": (C.c_int, [I32, I32, I32, P, P, P, P, P, P, P, F32, P, P, P, P]),
    "epsr_sumgr": (C.c_int, [I32, I32, P, I32, P, C.c_double, C.c_double, P, P, P, P, P, P]),
    "epsr_sumsq": (C.c_int, [I32, I32, P, I32, C.c_double, C.c_double, P, P, P, P, P]),
    "epsr_generate_ep": (C.c_int, [I32, I32, I32, I32, P, P, I32, I32, P, F32, P, P, P, P, P, P, P, I32, P, F32, F32,
                                   F32, F32, P, I32, P, P]),
    "epsr_ep_update": (C.c_int, [I32, I32, I32, P, I32, I32, P, P, P, P, I32, F32, P]),
    "epsr_pack_tables": (C.c_int, [I32, I32, P, P, P, P, P, P]),
    "epsr_en_mole_intra": (C.c_int, [P, P, P, P]),
    "epsr_minimage_centres": (C.c_int, [P, P]),
    "epsr_molfit_shake_scratch_bytes": (I64, [I32, I32]),
    "epsr_molfit_shake": (C.c_int, [P, P, P, P, F32, P, P, P, I64, P]),
    "epsr_generate_rp": (C.c_int, [P]),
    "epsr_calc_pwrexpr_grad": (C.c_int, [I32, I32, F32, F32, F32, F32, F32, P, P, F32, P, F32, F32]),
    "epsr_calc_gaussr_grad": (C.c_int, [I32, I32, F32, F32, F32, F32, P, P, F32, P, F32, F32]),
    "epsr_stog": (C.c_int, [F32, P, I32, P, P, I32, I32, P, P, P, P, P, I64, P]),
    "epsr_stog_scratch_bytes": (I64, [I32, I32]),
    "epsr_fit_expansion": (C.c_int, [P, P, P, P, P, P, I32, I32, I32, I32, I32, I32, P, P, I64, I32, P, P]),
    "epsr_fit_expansion_batch": (C.c_int, [I32, P, P, P, P, P, P, I32, I32, I32, I32, I32, I32, P, P, I64, I32, P,
                                           P]),
    "epsr_fit_expansion_batch_scratch_bytes": (I64, [I32, I32, I32]),
    "epsr_fit_expansion_scratch_bytes": (I64, [I32, I32]),
    "epsr_iteration_scratch_bytes": (I64, [C.POINTER(Iteration)]),
    "epsr_iteration_step": (C.c_int, [C.POINTER(Iteration), C.POINTER(IterationReport), P]),
}

_lib = None


def exported_symbols():
    """Names of every entry point the header declares (checked by the CPU test suite)."""
    return sorted(_SIGS)


def load(require_device=False):
    """Load the library (raising if it is missing); optionally require an sm_100 device."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIBPATH):
            raise EpsrGpuError(-1, f"{LIBPATH} is missing; run epsr_python_translation_b200.csrc.build")
        lib = C.CDLL(LIBPATH)
        for name, (res, args) in _SIGS.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    if require_device:
        global _device_ok
        if _device_ok is None:
            _device_ok = _lib.epsr_device_count() > 0
        if not _device_ok:
            raise EpsrGpuError(-1, "no sm_100 (B200) device visible")
    return _lib


_device_ok = None


def check(rc):
    if rc != 0:
        raise EpsrGpuError(rc, load().epsr_last_error().decode(errors="replace"))
    return rc
