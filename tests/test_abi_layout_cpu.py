"""The ctypes views of the C ABI's structs (epsr_python_translation_b200/_lib.py, batch.py)
against include/epsr_gpu.h itself: a small C program compiled with gcc prints each struct's
size and every field's offset as the header lays them out, and the Python side must agree,
so a field added to the header without its ctypes twin (or the other way round) fails here
rather than as a corrupted argument on the device."""

import ctypes as C
import os
import shutil
import subprocess

import pytest

from epsr_python_translation_b200 import _lib, batch

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

STRUCTS = [
    (_lib.Box, "epsr_box_t"), (_lib.Cells, "epsr_cells_t"), (_lib.Store, "epsr_store_t"), (_lib.Mc, "epsr_mc_t"),
    (_lib.Mlp, "epsr_mlp_t"), (_lib.Intra, "epsr_intra_t"), (_lib.Rp, "epsr_rp_t"),
    (_lib.Iteration, "epsr_iteration_t"), (_lib.IterationReport, "epsr_iteration_report_t"),
    (batch.BoxDesc, "epsr_bmc_box_t"), (batch.Bmc, "epsr_bmc_t"), (batch.BmcHist, "epsr_bmc_hist_t"),
]


def _c_layout(tmp_path):
    lines = ["#include <stdio.h>", "#include <stddef.h>", '#include "epsr_gpu.h"', "int main(void) {"]
    for cls, cname in STRUCTS:
        lines.append(f'    printf("{cname} size %zu\\n", sizeof({cname}));')
        for name, _ in cls._fields_:
            lines.append(f'    printf("{cname} {name} %zu\\n", offsetof({cname}, {name}));')
    lines += ["    return 0;", "}"]
    src = tmp_path / "layout.c"
    exe = tmp_path / "layout"
    src.write_text("\n".join(lines) + "\n")
    subprocess.run(["gcc", "-std=c11", "-I", os.path.join(ROOT, "include"), "-o", str(exe), str(src)], check=True,
                   capture_output=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    lay = {}
    for ln in out.splitlines():
        cname, key, val = ln.split()
        lay[(cname, key)] = int(val)
    return lay


@pytest.mark.skipif(shutil.which("gcc") is None, reason="needs gcc")
def test_ctypes_structs_match_the_header(tmp_path):
    lay = _c_layout(tmp_path)
    bad = []
    for cls, cname in STRUCTS:
        if C.sizeof(cls) != lay[(cname, "size")]:
            bad.append(f"{cname}: size {C.sizeof(cls)} (ctypes) vs {lay[(cname, 'size')]} (header)")
        for name, _ in cls._fields_:
            off = getattr(cls, name).offset
            if off != lay[(cname, name)]:
                bad.append(f"{cname}.{name}: offset {off} (ctypes) vs {lay[(cname, name)]} (header)")
    assert not bad, "\n".join(bad)
