"""Stage the reference's own Python solver into baseline/_ref/pythonHipims.

BENCHMARK AND TEST INFRASTRUCTURE ONLY.  The reference tree is not a
pip-installable project (no setup.py or pyproject.toml at its root, so
`pip install --target baseline/_ref <reference>` stops with "not installable"),
so this recipe does what that install would do for the two solver modules the
drop-in boundary serves: it copies CHANS-HiPIMS/hipims/pythonHipims/SWE_CUDA.py
(the `Godunov` class) and Parallel_SWE_CUDA.py byte for byte, unmodified, into
the git-ignored baseline/_ref/pythonHipims/.  That folder travels with the
repository snapshot (like baseline/_ref/libhipims_ref_cuda.so), so a machine
without the reference tree can run the reference solver class on this
library's op modules (baseline/ref_loop.py).

Usage: python baseline/install_ref_py.py [--ref REFERENCE_ROOT]
(default: $HIPIMS_REFERENCE_ROOT, else the reference checkout this recipe
was written against).
"""
from __future__ import annotations

import argparse
import hashlib
import os
import shutil
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT_DIR = os.path.join(HERE, "_ref", "pythonHipims")
DEFAULT_REF = os.environ.get("HIPIMS_REFERENCE_ROOT", "/root/reference")
PY_DIR = os.path.join("CHANS-HiPIMS", "hipims", "pythonHipims")
FILES = ("SWE_CUDA.py", "Parallel_SWE_CUDA.py")


def install(ref: str = DEFAULT_REF, quiet: bool = False) -> str | None:
    """Copy the solver modules; returns the output folder, or None when the
    reference tree is absent."""
    src_dir = os.path.join(ref, PY_DIR)
    if not all(os.path.isfile(os.path.join(src_dir, f)) for f in FILES):
        if not quiet:
            print(f"reference solver not found under {src_dir}", file=sys.stderr)
        return None
    os.makedirs(OUT_DIR, exist_ok=True)
    manifest = []
    for f in FILES:
        src, dst = os.path.join(src_dir, f), os.path.join(OUT_DIR, f)
        shutil.copyfile(src, dst)
        with open(dst, "rb") as fh:
            manifest.append(f"{hashlib.sha256(fh.read()).hexdigest()}  {f}")
    with open(os.path.join(OUT_DIR, "SHA256SUMS"), "w") as fh:
        fh.write("\n".join(manifest) + "\n")
    return OUT_DIR


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=DEFAULT_REF)
    out = install(ap.parse_args().ref)
    if out is None:
        sys.exit(1)
    print(out)
