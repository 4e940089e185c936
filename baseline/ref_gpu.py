"""The reference's own HiPIMS kernels on the GPU, as an ops object for the
Godunov loop: the plain FP64 GPU path the fused step is compared with.

BENCHMARK INFRASTRUCTURE ONLY.  baseline/build_ref_cuda.py builds
baseline/_ref/libhipims_ref_cuda.so from the reference's kernel sources; this
module binds its launchers with ctypes and exposes them under the op names of
hipims_b200.ops, so that ``Godunov(..., ops_impl=RefGpuOps())`` runs the
reference solver's step order (HP/SWE_CUDA.py:339-424, 497-502, 780-831) on
the reference's own device code.  The dt reduction is torch.min, as in the
reference (HP/SWE_CUDA.py:818-820).
"""
from __future__ import annotations

import ctypes
import os

import torch

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_ref", "libhipims_ref_cuda.so")

_P, _I = ctypes.c_void_p, ctypes.c_int


def available() -> bool:
    return os.path.exists(LIB)


class RefGpuOps:
    """Op functions of hipims_b200.ops backed by the reference's kernels (FP64)."""

    def __init__(self):
        if not available():
            raise FileNotFoundError(f"{LIB} is not built (python baseline/build_ref_cuda.py)")
        L = ctypes.CDLL(LIB)
        L.refgpu_flux2.argtypes = [_I] * 8 + [_P] * 17 + [_P]
        L.refgpu_flux1.argtypes = [_I] * 8 + [_P] * 17 + [_P]
        L.refgpu_friction_update.argtypes = [_I] + [_P] * 13 + [_P]
        L.refgpu_timestep.argtypes = [_I] + [_P] * 10 + [_P]
        L.refgpu_rain_station.argtypes = [_I] + [_P] * 4 + [_P]
        L.refgpu_flux_mask.argtypes = [_I] + [_P] * 4 + [_P]
        for f in ("refgpu_flux2", "refgpu_flux1", "refgpu_friction_update", "refgpu_timestep",
                  "refgpu_rain_station", "refgpu_flux_mask"):
            getattr(L, f).restype = _I
        self._L = L

    @staticmethod
    def _p(*ts):
        for t in ts:
            if t.is_floating_point() and t.dtype != torch.float64:
                raise TypeError("the reference kernels are bound in FP64 only")
        return [t.data_ptr() for t in ts]

    @staticmethod
    def _stream() -> int:
        return torch.cuda.current_stream().cuda_stream

    @staticmethod
    def _ok(rc: int, what: str) -> None:
        if rc != 0:
            raise RuntimeError(f"{what}: CUDA error {rc}")

    def flux_mask(self, fluxMask, h, index, t):
        self._ok(self._L.refgpu_flux_mask(h.numel(), *self._p(fluxMask, h, index, t),
                                          self._stream()), "fluxMask")

    def _flux(self, fn, wetMask, h_flux, qx_flux, qy_flux, h, wl, z, qx, qy, index, normal,
              given_depth, given_wl, given_q, dx, t, dt):
        dh, dw = given_depth.shape
        wh, ww = given_wl.shape
        qh, qw = given_q.shape
        self._ok(fn(
            wetMask.numel(), h.numel(), dw, dh, ww, wh, qw, qh,
            *self._p(wetMask, h, wl, z, qx, qy, index, normal, given_depth, given_wl,
                     given_q, dx, t, dt, h_flux, qx_flux, qy_flux), self._stream()), "addFlux")

    def flux_2nd_order(self, *args):
        """HC/flucCal_2ndOrder_jh_improved_Kernel.cu (MUSCL + hydrostatic + HLLC)."""
        self._flux(self._L.refgpu_flux2, *args)

    def flux_1st_order(self, *args):
        """HC/fluxCal_jh_modified_surface_Kernel.cu (bed-only minmod + HLLC), the
        scheme of the coupled server (CHANS-HiPIMS_server.py: secondOrder False)."""
        self._flux(self._L.refgpu_flux1, *args)

    def friction_update(self, wetMask, h_update, qx_update, qy_update, z_update, landuse, h,
                        wl, qx, qy, z, manning, dt):
        self._ok(self._L.refgpu_friction_update(
            wetMask.numel(), *self._p(wetMask, h_update, qx_update, qy_update, z_update,
                                      landuse, h, wl, qx, qy, z, manning, dt),
            self._stream()), "addFriction_eulerUpdate")

    def update_timestep(self, wetMask, accelerator, h_max, h, qx, qy, dx, CFL, t, dt):
        self._ok(self._L.refgpu_timestep(
            wetMask.numel(), *self._p(wetMask, h_max, h, qx, qy, accelerator, dx, CFL, t, dt),
            self._stream()), "updateTimestep")

    def station_rain(self, h_update, rainStationMask, rainStationData, dt):
        self._ok(self._L.refgpu_rain_station(
            rainStationMask.numel(), *self._p(h_update, rainStationMask, rainStationData, dt),
            self._stream()), "addStation_Precipitation")

    @staticmethod
    def device_min(x, out=None):
        return torch.min(x).reshape(1)

    def infiltration(self, *args):
        raise NotImplementedError("the reference infiltration kernel is not bound here")

    def euler_update(self, *args):
        raise NotImplementedError("the reference Euler kernel is not bound here")
