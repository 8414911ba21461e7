"""The C ABI library builds, loads without a GPU and exports every declared entry point;
without a device the product path fails loudly instead of falling back to the CPU."""

import ctypes as C
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "epsr_gpu.h")


def declared():
    txt = open(HEADER).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(epsr_[a-z0-9_]+)\s*\(", txt)))


@pytest.fixture(scope="module")
def lib():
    from epsr_python_translation_b200.csrc import build
    path = build.build()
    return C.CDLL(path)


def test_header_declares_entry_points():
    names = declared()
    assert "epsr_molfit" in names and "epsr_atogen" in names and len(names) >= 20


def test_library_exports_every_declared_symbol(lib):
    for name in declared():
        assert hasattr(lib, name), name


def test_python_binding_covers_header():
    from epsr_python_translation_b200 import _lib
    assert set(declared()) <= set(_lib.exported_symbols())


def test_host_only_entry_points_run_without_gpu(lib):
    lib.epsr_version.restype = C.c_char_p
    assert b"sm_100a" in lib.epsr_version()
    dims = np.zeros(4, np.int32)
    lat6 = np.array([1, 0, 0, 1, 0, 1], np.float32)
    rc = lib.epsr_cell_dims(10, 600, lat6.ctypes.data_as(C.c_void_p), dims.ctypes.data_as(C.c_void_p))
    assert rc == 0 and list(dims) == [5, 5, 5, 125]
    # null pointers are rejected with a status, not a crash
    assert lib.epsr_cell_dims(10, 600, None, None) == 1


def test_cell_dims_match_oracle_on_golden_cases():
    from oracle import oracle
    from tests import goldens
    from epsr_python_translation_b200 import _lib
    L = _lib.load()
    for case in goldens.CASES:
        z = goldens.load(case)
        nmol = int(z["sys_naf"].shape[0])
        dims = np.zeros(4, np.int32)
        lat6 = np.array([1, 0, 0, 1, 0, 1], np.float32)
        assert L.epsr_cell_dims(int(z["in_nmolcell"]), nmol, lat6.ctypes.data_as(C.c_void_p),
                                dims.ctypes.data_as(C.c_void_p)) == 0
        assert dims[3] == int(z["cell_ncell"]), case


def test_device_path_refuses_without_gpu():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from epsr_python_translation_b200 import _lib
    from epsr_python_translation_b200.box import BoxArrays
    from tests import goldens
    with pytest.raises(_lib.EpsrGpuError):
        from epsr_python_translation_b200.device import DeviceBox
        DeviceBox(BoxArrays.from_golden(goldens.load("c1_water")))


def _zero_args(argtypes):
    vals = []
    for a in argtypes:
        if a in (C.c_float, C.c_double):
            vals.append(a(0.0))
        elif a in (C.c_int8, C.c_int16, C.c_int32, C.c_int64, C.c_uint32, C.c_uint64, C.c_size_t):
            vals.append(a(0))
        else:
            vals.append(None)
    return vals


def test_every_entry_point_rejects_null_and_zero_arguments():
    """Each status-returning entry point, given null pointers and zero sizes, returns the
    argument-error status with a message naming the entry -- checked before any CUDA call, so
    no GPU is needed and nothing is dereferenced."""
    from epsr_python_translation_b200 import _lib
    L = _lib.load()
    checked = 0
    for name, (restype, argtypes) in _lib._SIGS.items():
        if not argtypes or name.endswith("_bytes") or name in ("epsr_last_error", "epsr_timing_enable"):
            continue
        rc = getattr(L, name)(*_zero_args(argtypes))
        assert rc == 1, (name, rc)
        msg = L.epsr_last_error().decode()
        assert name in msg, (name, msg)
        checked += 1
    assert checked >= 25


def test_atogen_refuses_too_many_atom_types_before_device_work():
    """More than 64 atom types is refused by epsr_atogen (and so by epsr_atogen_noalloc) before
    any memset or ran1 draw: the check runs before any CUDA call, so no GPU is needed, and a
    ran1 state handed in is left as it was."""
    from epsr_python_translation_b200 import _lib
    L = _lib.load()
    b = _lib.Box()
    b.nmol, b.natom, b.npairs, b.ntype, b.nmoltype = 100, 300, 65 * 66 // 2, 65, 1
    b.ld = 101
    ngr = np.array([1000], np.int32)
    buf = np.zeros(64, np.float32)
    p = buf.ctypes.data_as(C.c_void_p)
    ran1 = np.arange(35, dtype=np.int32)
    before = ran1.copy()
    rc = L.epsr_atogen(C.byref(b), 100, 1.0, 30.0, p, p, p, p, p, 3, ngr.ctypes.data_as(C.c_void_p),
                       ran1.ctypes.data_as(C.c_void_p), p, 101, p, p, p, 1 << 30, None)
    assert rc == 4   # EPSR_ERR_UNSUPPORTED
    assert "64 atom types" in L.epsr_last_error().decode()
    assert np.array_equal(ran1, before)
