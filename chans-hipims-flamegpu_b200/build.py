"""Build libhipims_b200.so (sm_100a) in-tree with nvcc.

    python chans-hipims-flamegpu_b200/build.py [--verbose] [--ptxas]

Each source is compiled for -gencode arch=compute_100a,code=sm_100a with
-lineinfo; object files go to chans-hipims-flamegpu_b200/_build/ and the
shared library to chans-hipims-flamegpu_b200/libhipims_b200.so.  The CUDA
runtime is linked statically so the library does not depend on which
libcudart the host process loaded.
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libhipims_b200.so")
INCLUDE = os.path.join(ROOT, "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
          "-I", INCLUDE, "-I", CSRC]
# Per-source numerics flags.  The compat ops follow the reference's FP64
# operation order, so no FMA contraction there; the fused FP32 path uses
# approximate single-precision division/sqrt (double is unaffected).
PER_FILE = {
    "hb_compat.cu": ["-fmad=false"],
    "hb_fused.cu": ["-ftz=true", "-prec-div=false", "-prec-sqrt=false"],
}
SOURCES = ["hb_abi.cpp", "hb_compat.cu", "hb_fused.cu", "hb_adjoint.cu"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise FileNotFoundError("nvcc not found")


def _stale(obj: str, deps: list[str]) -> bool:
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, ptxas: bool = False, force: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    headers += [os.path.join(INCLUDE, f) for f in os.listdir(INCLUDE) if f.endswith(".h")]
    objs = []
    cc = nvcc()
    for src in SOURCES:
        path = os.path.join(CSRC, src)
        obj = os.path.join(BUILD, src + ".o")
        objs.append(obj)
        if not force and not _stale(obj, [path, *headers, __file__]):
            continue
        cmd = [cc, *ARCH, *COMMON, *PER_FILE.get(src, []), "-c", path, "-o", obj]
        if ptxas and src.endswith(".cu"):
            cmd += ["-Xptxas", "-v"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    if force or _stale(LIB, objs):
        cmd = [cc, *ARCH, "-shared", "-cudart", "static", "-o", LIB, *objs]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--ptxas", action="store_true")
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    print(build(a.verbose, a.ptxas, a.force))
    sys.exit(0)
