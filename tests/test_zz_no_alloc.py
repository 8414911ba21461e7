"""epsr_atogen_noalloc (working memory in a file-scope device array) against epsr_atogen
(caller scratch): identical histograms, potex, sample counts and ran1 state on two calls in
a row.  The histograms are integer counts normalised in float32, so the tolerance is zero:
bit-identical.  This file is collected last so that it also runs after every other test has
used the device."""

import ctypes as C

import numpy as np
import pytest
import torch

from epsr_python_translation_b200 import _lib
from epsr_python_translation_b200.box import BoxArrays, Ran1State
from tests import goldens
from tests.goldens import assert_bits_equal

f32 = np.float32


def _noalloc(d, ngrsamples, ran1_t, rminex, ycoh=None):
    """One epsr_atogen_noalloc call on DeviceBox d; returns (ngr, wav, potex) on the host."""
    b = d.host
    ld = b.npt + 1
    wav = torch.zeros(2 * b.npairs * ld, dtype=torch.float32, device=d.dev)
    potex = torch.zeros(b.npairs, dtype=torch.float32, device=d.dev)
    rmx = torch.from_numpy(np.asarray(rminex, f32)).to(d.dev)
    yc = torch.from_numpy(np.zeros(ld, f32) if ycoh is None else np.asarray(ycoh, f32)[:ld].copy()).to(d.dev)
    ngr = np.array([ngrsamples], np.int32)
    p = lambda t: C.c_void_p(t.data_ptr())  # noqa: E731
    _lib.check(d.lib.epsr_atogen_noalloc(C.byref(d.cbox), b.npt1, 1.0, float(b.dmax), p(rmx), p(d.cfrac), p(yc),
                                         p(d.n1extr), p(d.n2extr), b.natomr, ngr.ctypes.data_as(C.c_void_p),
                                         p(ran1_t), p(wav), ld, p(potex),
                                         C.c_void_p(torch.cuda.current_stream().cuda_stream)))
    torch.cuda.synchronize()
    return int(ngr[0]), wav.cpu().numpy(), potex.cpu().numpy()


def _boxes():
    out = []
    for case in ("c1_water", "mix_small"):
        z = goldens.load(case)
        box = BoxArrays.from_golden(z)
        last = int(z["mf_cycles"]) - 1
        for k in ("xa", "ya", "za", "xadd", "yadd", "zadd"):
            setattr(box, k, z[f"mf{last}_{k}"].copy())
        out.append((case, box, Ran1State.from_golden(z, "ag_ran1_before_"), int(z["ag_ngrsamples_in"]),
                    z["ag_rminex"], None, z))
    from epsr_python_translation_b200.configs import make_workload
    wl = make_workload("c2_mixture")
    box = BoxArrays.from_system(wl.system)
    out.append(("c2_mixture", box, Ran1State(idum=-12345), wl.ngrsamples, np.full(box.npairs, f32(-2.0), f32),
                wl.ycoh, None))
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("which", [0, 1, 2])
def test_noalloc_atogen_matches_scratch_entry_two_calls(which):
    from epsr_python_translation_b200.device import DeviceBox
    case, box, r0, ngrs, rminex, ycoh, z = _boxes()[which]
    d = DeviceBox(box)
    ta = d.ran1_tensor(r0)
    tb = d.ran1_tensor(r0)
    for call in range(2):
        ngr_a = d.atogen(ngrs, ta, rminex, ycoh=ycoh)
        wav_a, potex_a = d.download_wav()
        ngr_b, wav_b, potex_b = _noalloc(d, ngrs, tb, rminex, ycoh=ycoh)
        assert ngr_b == ngr_a, (case, call)
        assert_bits_equal(wav_b.reshape(wav_a.shape), wav_a, f"{case} wav call {call}")
        assert_bits_equal(potex_b, potex_a, f"{case} potex call {call}")
        assert np.array_equal(tb.cpu().numpy(), ta.cpu().numpy()), (case, call)
        assert d.last_pair_updates > 0
        if call == 0 and z is not None:     # the first call also reproduces the reference
            mine = wav_b.reshape(2, box.npairs, box.npt + 1)[:, :, 1:box.npt1 + 1].transpose(0, 2, 1)
            assert_bits_equal(mine, z["ag_wav"], f"{case} wav vs reference")


def test_noalloc_atogen_rejects_oversize_box_before_device_work():
    """The size check runs before any CUDA call, so it is exercised without a GPU."""
    lib = _lib.load(require_device=False)
    b = _lib.Box()
    b.nmol, b.natom, b.npairs, b.ntype, b.nmoltype = 60000, 180000, 3, 2, 1
    ngr = np.array([1000], np.int32)
    rc = lib.epsr_atogen_noalloc(C.byref(b), 100, 1.0, 30.0, None, None, None, None, None, 3,
                                 ngr.ctypes.data_as(C.c_void_p), None, None, 101, None, None)
    assert rc == 3   # EPSR_ERR_CAPACITY
    msg = lib.epsr_last_error().decode()
    assert "epsr_atogen_noalloc" in msg and "50000" in msg and "use epsr_atogen" in msg
    b.nmol, b.natom, b.npairs = 100, 300, 600
    rc = lib.epsr_atogen_noalloc(C.byref(b), 500, 1.0, 30.0, None, None, None, None, None, 3,
                                 ngr.ctypes.data_as(C.c_void_p), None, None, 501, None, None)
    assert rc == 3 and "histogram" in lib.epsr_last_error().decode()
