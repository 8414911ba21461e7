"""Build libepsr_gpu.so (sm_100a) in-tree with nvcc.

    python -m epsr_python_translation_b200.csrc.build [--verbose]

The library is written next to the package (``epsr_python_translation_b200/libepsr_gpu.so``)
so that it travels with the source tree.  -fmad=false keeps every float32 expression
uncontracted; the bit-exact paths also use explicit round-to-nearest intrinsics.
"""

from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.dirname(HERE)
ROOT = os.path.dirname(PKG)
LIB = os.path.join(PKG, "libepsr_gpu.so")
SOURCES = ["abi.cu", "ran1.cu", "cells.cu", "store.cu", "mc.cu", "atogen.cu", "transforms.cu", "fitexp.cu",
           "mc_spec.cu", "press.cu", "iteration.cu", "sums.cu", "ep.cu", "shake.cu", "rp.cu", "mlp.cu", "batch.cu"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-fmad=false", "-std=c++17",
         "-Xcompiler", "-fPIC", "-I", os.path.join(ROOT, "include")]


def sources():
    return [os.path.join(HERE, s) for s in SOURCES if os.path.exists(os.path.join(HERE, s))]


def needs_build():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = sources() + [os.path.join(HERE, "common.cuh"), os.path.join(ROOT, "include", "epsr_gpu.h")]
    deps += [os.path.join(HERE, f) for f in os.listdir(HERE) if f.endswith(".cuh")]
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(verbose=False, force=False):
    if not force and not needs_build():
        return LIB
    objdir = os.path.join(ROOT, "_build")
    os.makedirs(objdir, exist_ok=True)
    objs = []
    for src in sources():
        obj = os.path.join(objdir, os.path.basename(src) + ".o")
        cmd = [NVCC, *FLAGS, "-c", src, "-o", obj]
        if verbose:
            cmd += ["-Xptxas", "-v"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if verbose or r.returncode:
            sys.stderr.write(r.stdout + r.stderr)
        if r.returncode:
            raise RuntimeError(f"nvcc failed on {src}")
        objs.append(obj)
    tmp = LIB + ".tmp"
    cmd = [NVCC, "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-Xcompiler", "-fPIC", "-o", tmp, *objs]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("link failed")
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(verbose="--verbose" in sys.argv, force=True)
    print(LIB)
