"""Build recipe for libdgv_b200.so (sm_100a).

Every source is compiled with nvcc for `-gencode arch=compute_100a,code=sm_100a`
and linked into one shared library in this package directory, so that it
travels with the source tree.  The CUDA runtime is linked statically: the
library has no dependency on PyTorch or on the runtime version torch bundles.

Per-file flags:
  synth.cu, stepping.cu  -fmad=false  (bit-reproducible prefilter/values and
                                        the reference's stage arithmetic)
  host code               -ffp-contract=off (node coordinates bit for bit)
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libdgv_b200.so")
BUILD = os.path.join(HERE, "_build")

SOURCES = [
    ("grid.cpp", []),
    ("layout.cpp", []),
    ("afile.cpp", []),
    ("api.cu", []),
    ("collide.cu", []),
    ("collide_tc.cu", []),
    ("adjoint.cu", []),
    ("noalloc.cu", []),
    ("synth.cu", ["-fmad=false"]),
    ("seta.cu", ["-fmad=false"]),
    ("stepping.cu", ["-fmad=false"]),
    ("group.cu", []),
]

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-ffp-contract=off",
          "-I" + os.path.join(HERE, "..", "include")]


def nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _stale(obj: str, deps) -> bool:
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, force: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    nv = nvcc()
    headers = [os.path.join(CSRC, h) for h in os.listdir(CSRC) if h.endswith((".h", ".cuh"))]
    headers.append(os.path.join(HERE, "..", "include", "dgv_b200.h"))
    objs = []
    for src, extra in SOURCES:
        path = os.path.join(CSRC, src)
        obj = os.path.join(BUILD, src + ".o")
        objs.append(obj)
        if not force and not _stale(obj, [path] + headers):
            continue
        lang = ["-x", "cu"] if src.endswith(".cu") else []
        cmd = [nv] + ARCH + COMMON + extra + lang + ["-c", path, "-o", obj]
        if verbose:
            cmd += ["-Xptxas", "-v"]
            print(" ".join(cmd))
        subprocess.check_call(cmd)
    if force or _stale(OUT, objs):
        cmd = [nv] + ARCH + ["-shared", "-cudart", "static", "-o", OUT] + objs
        if verbose:
            print(" ".join(cmd))
        subprocess.check_call(cmd)
    return OUT


if __name__ == "__main__":
    build(verbose="-v" in sys.argv, force="-f" in sys.argv)
    print(OUT)
