"""Build the reference's own HiPIMS kernels for the B200 (sm_100a) as a plain
FP64 GPU baseline.

BENCHMARK INFRASTRUCTURE ONLY.  Output: baseline/_ref/libhipims_ref_cuda.so
(git-ignored; it travels with the repository snapshot as a built file).

Recipe: each reference kernel file is read where it lies under the reference
tree, the text up to its torch launcher is kept, its #include lines are
dropped, and the result is piped to nvcc on stdin with baseline/ref_cuda_shim.h
and a launcher of our own appended.  The launchers use the reference's own
launch shapes (512-thread blocks for the flux and flux-mask kernels,
gpu.cuh's 1024-thread blocks for the others).  No reference source is written
anywhere; the torch launchers are never compiled, so the reference's 2-rule
torch patch is not needed.

Usage: python baseline/build_ref_cuda.py [--ref REFERENCE_ROOT]
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT_DIR = os.path.join(HERE, "_ref")
LIB = os.path.join(OUT_DIR, "libhipims_ref_cuda.so")
# the reference checkout: $HIPIMS_REFERENCE_ROOT, else where this recipe was written
DEFAULT_REF = os.environ.get("HIPIMS_REFERENCE_ROOT", "/root/reference")
KERNEL_DIR = os.path.join("CHANS-HiPIMS", "hipims", "cuda")

_LAUNCH = {
    "flucCal_2ndOrder_jh_improved_Kernel.cu": (
        "void fluxCalculation_cuda(",
        r"""
extern "C" int refgpu_flux2(int M, int N, int dw, int dh, int ww, int wh, int qw, int qh,
    int32_t *wet, double *h, double *wl, double *z, double *qx, double *qy,
    int32_t *index, double *normal, double *gd, double *gw, double *gq,
    double *dx, double *t, double *dt, double *hf, double *qxf, double *qyf, void *st) {
  if (M == 0) return 0;
  fluxCalculation_kernel<double><<<(M + 512 - 1) / 512, 512, 0, (cudaStream_t)st>>>(
      M, N, dw, dh, ww, wh, qw, qh, wet, h, wl, z, qx, qy, index, normal, gd, gw, gq,
      dx, t, dt, hf, qxf, qyf);
  return (int)cudaGetLastError();
}
""",
    ),
    # the 1st-order flux kernel has the 2nd-order one's name: renamed in its
    # translation unit (PREFIX below) so that the two launch stubs stay apart
    "fluxCal_jh_modified_surface_Kernel.cu": (
        "void fluxCalculation_cuda(",
        r"""
extern "C" int refgpu_flux1(int M, int N, int dw, int dh, int ww, int wh, int qw, int qh,
    int32_t *wet, double *h, double *wl, double *z, double *qx, double *qy,
    int32_t *index, double *normal, double *gd, double *gw, double *gq,
    double *dx, double *t, double *dt, double *hf, double *qxf, double *qyf, void *st) {
  if (M == 0) return 0;
  fluxCalculation_kernel<double><<<(M + 512 - 1) / 512, 512, 0, (cudaStream_t)st>>>(
      M, N, dw, dh, ww, wh, qw, qh, wet, h, wl, z, qx, qy, index, normal, gd, gw, gq,
      dx, t, dt, hf, qxf, qyf);
  return (int)cudaGetLastError();
}
""",
    ),
    "friction_implicit_andUpdate_jh_Kernel.cu": (
        "void frictionCalculation_cuda(",
        r"""
extern "C" int refgpu_friction_update(int M, int32_t *wet, double *hu, double *qxu,
    double *qyu, double *zu, uint8_t *landuse, double *h, double *wl, double *qx,
    double *qy, double *z, double *manning, double *dt, void *st) {
  if (M == 0) return 0;
  frictionCalculation_kernel<double><<<GET_BLOCKS(M), CUDA_NUM_THREADS, 0,
                                       (cudaStream_t)st>>>(
      M, wet, hu, qxu, qyu, zu, landuse, h, wl, qx, qy, z, manning, dt);
  return (int)cudaGetLastError();
}
""",
    ),
    "timeControl_Kernel.cu": (
        "void timeControl_cuda(",
        r"""
extern "C" int refgpu_timestep(int M, int32_t *wet, double *h_max, double *h, double *qx,
    double *qy, double *accel, double *dx, double *cfl, double *t, double *dt, void *st) {
  if (M == 0) return 0;
  timeControl_accer<double><<<GET_BLOCKS(M), CUDA_NUM_THREADS, 0, (cudaStream_t)st>>>(
      M, wet, h_max, h, qx, qy, accel, dx, cfl, t, dt);
  return (int)cudaGetLastError();
}
""",
    ),
    "stationPrecipitation_Kernel.cu": (
        "void station_PrecipitationCalculation_cuda(",
        r"""
extern "C" int refgpu_rain_station(int N, double *hu, int16_t *mask, double *data,
    double *dt, void *st) {
  if (N == 0) return 0;
  station_PrecipitationCalculation_kernel<double><<<GET_BLOCKS(N), CUDA_NUM_THREADS, 0,
                                                    (cudaStream_t)st>>>(N, hu, mask, data, dt);
  return (int)cudaGetLastError();
}
""",
    ),
    "fluxMaskGenerator_Kernel.cu": (
        "void fluxMask_cuda(",
        r"""
extern "C" int refgpu_flux_mask(int N, bool *out, double *h, int32_t *index, double *t,
    void *st) {
  if (N == 0) return 0;
  fluxMask_kernel<double><<<(N + 512 - 1) / 512, 512, 0, (cudaStream_t)st>>>(
      N, out, h, index, t);
  return (int)cudaGetLastError();
}
""",
    ),
}

PREFIX = {
    "fluxCal_jh_modified_surface_Kernel.cu":
        "#define fluxCalculation_kernel refgpu_first_order_fluxCalculation_kernel\n",
}

NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17",
              "-Xcompiler", "-fPIC", "-w"]


def _kernel_text(path: str, marker: str) -> str:
    with open(path, "r", encoding="utf-8") as f:
        src = f.read()
    cut = src.find(marker)
    if cut < 0:
        raise RuntimeError(f"launcher marker {marker!r} not found in {path}")
    return "\n".join(ln for ln in src[:cut].splitlines()
                     if not ln.lstrip().startswith("#include"))


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise FileNotFoundError("nvcc not found")


def build(ref_root: str = DEFAULT_REF, verbose: bool = False, ptxas: bool = False) -> str:
    kdir = os.path.join(ref_root, KERNEL_DIR)
    if not os.path.isdir(kdir):
        raise FileNotFoundError(f"reference kernels not found under {kdir}")
    os.makedirs(OUT_DIR, exist_ok=True)
    objs = []
    cc = nvcc()
    for fname, (marker, launcher) in _LAUNCH.items():
        text = ('#include "ref_cuda_shim.h"\n' + PREFIX.get(fname, "") +
                _kernel_text(os.path.join(kdir, fname), marker))
        text += "\n" + launcher
        obj = os.path.join(OUT_DIR, os.path.splitext(fname)[0] + ".o")
        cmd = [cc, *NVCC_FLAGS, "-I", HERE, "-x", "cu", "-", "-c", "-o", obj]
        if ptxas:
            cmd += ["-Xptxas", "-v"]
        if verbose:
            print(" ".join(cmd), "<", fname, flush=True)
        subprocess.run(cmd, input=text.encode(), check=True)
        objs.append(obj)
    subprocess.run([cc, "-gencode", "arch=compute_100a,code=sm_100a", "-shared",
                    "-cudart", "static", "-o", LIB, *objs], check=True)
    for o in objs:
        os.remove(o)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=DEFAULT_REF)
    ap.add_argument("--ptxas", action="store_true")
    a = ap.parse_args()
    print(build(a.ref, verbose=True, ptxas=a.ptxas))
    sys.exit(0)
