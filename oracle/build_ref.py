"""Build the reference's own HiPIMS kernels for the host CPU.

TEST INFRASTRUCTURE ONLY.  Output: oracle/_ref/libhipims_ref_host.so (git-ignored,
travels with the repository snapshot as a built file).

Recipe: each reference kernel file is read where it lies under the reference
tree, the text up to its torch launcher (``void *_cuda(``) is kept, its
``#include`` lines are dropped, and the result is piped to g++ on stdin with
oracle/ref_shim.h force-included and a small host driver of our own appended.
No reference source is written anywhere; only object files and the shared
library land in oracle/_ref/.

The reference's kernels compile unchanged this way; the 2-rule torch patch is
not needed because the torch launchers are never compiled.

Usage: python oracle/build_ref.py [--ref REFERENCE_ROOT]
"""
from __future__ import annotations

import argparse
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT_DIR = os.path.join(HERE, "_ref")
LIB = os.path.join(OUT_DIR, "libhipims_ref_host.so")
# the reference checkout: $HIPIMS_REFERENCE_ROOT, else where this recipe was written
DEFAULT_REF = os.environ.get("HIPIMS_REFERENCE_ROOT", "/root/reference")
KERNEL_DIR = os.path.join("CHANS-HiPIMS", "hipims", "cuda")

# Host drivers: one extern "C" entry per kernel.  Each loops over the kernel's
# thread index with OpenMP; scalar "tensors" (dx, t, dt, CFL) are passed as
# pointers exactly as the kernels expect them.
_DRIVERS = {
    "flucCal_2ndOrder_jh_improved_Kernel.cu": (
        "void fluxCalculation_cuda(",
        r"""
extern "C" void ref_flux2(int M, int N, int dw, int dh, int ww, int wh, int qw, int qh,
    int32_t *wet, double *h, double *wl, double *z, double *qx, double *qy,
    const int32_t *index, const double *normal, double *gd, double *gw, double *gq,
    double *dx, double *t, double *dt, double *hf, double *qxf, double *qyf) {
#pragma omp parallel for schedule(static)
  for (int w = 0; w < M; ++w) {
    blockIdx.x = 0; blockDim.x = 0; threadIdx.x = (unsigned)w;
    fluxCalculation_kernel<double>(M, N, dw, dh, ww, wh, qw, qh, wet, h, wl, z, qx, qy,
        index, normal, gd, gw, gq, dx, t, dt, hf, qxf, qyf);
  }
}
""",
    ),
    "fluxCal_jh_modified_surface_Kernel.cu": (
        "void fluxCalculation_cuda(",
        r"""
extern "C" void ref_flux1(int M, int N, int dw, int dh, int ww, int wh, int qw, int qh,
    int32_t *wet, double *h, double *wl, double *z, double *qx, double *qy,
    const int32_t *index, const double *normal, double *gd, double *gw, double *gq,
    double *dx, double *t, double *dt, double *hf, double *qxf, double *qyf) {
#pragma omp parallel for schedule(static)
  for (int w = 0; w < M; ++w) {
    blockIdx.x = 0; blockDim.x = 0; threadIdx.x = (unsigned)w;
    fluxCalculation_kernel<double>(M, N, dw, dh, ww, wh, qw, qh, wet, h, wl, z, qx, qy,
        index, normal, gd, gw, gq, dx, t, dt, hf, qxf, qyf);
  }
}
""",
    ),
    "friction_implicit_andUpdate_jh_Kernel.cu": (
        "void frictionCalculation_cuda(",
        r"""
extern "C" void ref_friction_update(int M, int32_t *wet, double *hu, double *qxu,
    double *qyu, double *zu, uint8_t *landuse, double *h, double *wl, double *qx,
    double *qy, double *z, double *manning, double *dt) {
#pragma omp parallel for schedule(static)
  for (int w = 0; w < M; ++w) {
    blockIdx.x = 0; blockDim.x = 0; threadIdx.x = (unsigned)w;
    frictionCalculation_kernel<double>(M, wet, hu, qxu, qyu, zu, landuse, h, wl, qx, qy,
        z, manning, dt);
  }
}
""",
    ),
    "timeControl_Kernel.cu": (
        "void timeControl_cuda(",
        r"""
extern "C" void ref_timestep(int M, int32_t *wet, double *h_max, double *h, double *qx,
    double *qy, double *accel, double *dx, double *cfl, double *t, double *dt) {
#pragma omp parallel for schedule(static)
  for (int w = 0; w < M; ++w) {
    blockIdx.x = 0; blockDim.x = 0; threadIdx.x = (unsigned)w;
    timeControl_accer<double>(M, wet, h_max, h, qx, qy, accel, dx, cfl, t, dt);
  }
}
""",
    ),
    "stationPrecipitation_Kernel.cu": (
        "void station_PrecipitationCalculation_cuda(",
        r"""
extern "C" void ref_rain_station(int N, double *hu, int16_t *mask, double *data,
    double *dt) {
#pragma omp parallel for schedule(static)
  for (int w = 0; w < N; ++w) {
    blockIdx.x = 0; blockDim.x = 0; threadIdx.x = (unsigned)w;
    station_PrecipitationCalculation_kernel<double>(N, hu, mask, data, dt);
  }
}
""",
    ),
    "fluxMaskGenerator_Kernel.cu": (
        "void fluxMask_cuda(",
        r"""
extern "C" void ref_flux_mask(int N, bool *out, double *h, const int32_t *index,
    double *t) {
#pragma omp parallel for schedule(static)
  for (int w = 0; w < N; ++w) {
    blockIdx.x = 0; blockDim.x = 0; threadIdx.x = (unsigned)w;
    fluxMask_kernel<double>(N, out, h, index, t);
  }
}
""",
    ),
    "euler_update_Kernel.cu": (
        "void euler_update_cuda(",
        r"""
extern "C" void ref_euler_update(int M, int32_t *mask, double *hu, double *qxu,
    double *qyu, double *zu, double *h, double *wl, double *z, double *qx, double *qy) {
#pragma omp parallel for schedule(static)
  for (int w = 0; w < M; ++w) {
    blockIdx.x = 0; blockDim.x = 0; threadIdx.x = (unsigned)w;
    euler_update_kernel<double>(M, mask, hu, qxu, qyu, zu, h, wl, z, qx, qy);
  }
}
""",
    ),
    "infiltrationCUDA_Kernel.cu": (
        "void infiltrationCalculation_cuda(",
        r"""
extern "C" void ref_infiltration(int M, int32_t *wet, double *hu, uint8_t *landuse,
    double *h, double *ks, double *psi, double *dth, double *cum, double *dt) {
#pragma omp parallel for schedule(static)
  for (int w = 0; w < M; ++w) {
    blockIdx.x = 0; blockDim.x = 0; threadIdx.x = (unsigned)w;
    infiltrationCalculation_kernel<double>(M, wet, hu, landuse, h, ks, psi, dth, cum, dt);
  }
}
""",
    ),
}

CXXFLAGS = ["-O2", "-fPIC", "-fopenmp", "-std=c++17", "-w"]


def _kernel_text(path: str, marker: str) -> str:
    with open(path, "r", encoding="utf-8") as f:
        src = f.read()
    cut = src.find(marker)
    if cut < 0:
        raise RuntimeError(f"launcher marker {marker!r} not found in {path}")
    body = [ln for ln in src[:cut].splitlines() if not ln.lstrip().startswith("#include")]
    return "\n".join(body)


def build(ref_root: str = DEFAULT_REF, verbose: bool = False) -> str:
    kdir = os.path.join(ref_root, KERNEL_DIR)
    if not os.path.isdir(kdir):
        raise FileNotFoundError(f"reference kernels not found under {kdir}")
    os.makedirs(OUT_DIR, exist_ok=True)
    objs = []
    for fname, (marker, driver) in _DRIVERS.items():
        text = '#include "ref_shim.h"\n' + _kernel_text(os.path.join(kdir, fname), marker)
        text += "\n" + driver
        obj = os.path.join(OUT_DIR, os.path.splitext(fname)[0] + ".o")
        cmd = ["g++", *CXXFLAGS, "-I", HERE, "-x", "c++", "-", "-c", "-o", obj]
        if verbose:
            print(" ".join(cmd), "<", fname)
        subprocess.run(cmd, input=text.encode(), check=True)
        objs.append(obj)
    cmd = ["g++", "-shared", "-fopenmp", "-o", LIB, *objs]
    subprocess.run(cmd, check=True)
    for o in objs:
        os.remove(o)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=DEFAULT_REF)
    a = ap.parse_args()
    print(build(a.ref, verbose=True))
    sys.exit(0)
