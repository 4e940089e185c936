"""Godunov: the reference solver's object API over the B200 compat ops.

Same constructor, method names, state attributes and step semantics as the
reference class ``Godunov`` (HP/SWE_CUDA.py:62-928), so drivers written
against it (``CHANS-HiPIMS_server.py:246-256``, ``HP/CatchFlood_main.py``) run
unchanged.  The step order is

    addFlux()                               fluxMask -> active list -> flux op
    addStation_PrecipitationSource(R, dev)  rain table interpolation -> rain op
    time_friction_euler_update_cuda(dev)    friction/update op -> timestep op
                                            -> min -> 10x cap -> export clip

Differences from the reference, all without effect on the numbers:
no ``torch.cuda.empty_cache()`` and no ``print`` per step; the min of the
CFL steps is taken on the device (ops.device_min); the export decision still
reads ``t`` and ``dt`` on the host once per step as the reference does.
"""
from __future__ import annotations

import os

import numpy as np
import torch

from . import ops
from .topology import compact_index


class Godunov:
    def __init__(self, device, dx, CFL, Export_timeStep, t=0.0, export_n=0,
                 secondOrder=False, firstTimeStep=1.0e-4, tensorType=torch.float64,
                 ops_impl=None):
        # ops_impl: an object with the op functions of hipims_b200.ops (default),
        # so that the same loop can drive another implementation of the ops
        self._ops = ops if ops_impl is None else ops_impl
        self._tensorType = tensorType
        self._secondOrder = secondOrder
        self._device = torch.device(device)
        self.dx = torch.tensor([dx], dtype=tensorType, device=device)
        self.cfl = torch.tensor([CFL], dtype=tensorType, device=device)
        self._manning = torch.tensor([0.0], dtype=tensorType, device=device)
        self.export_timeStep = Export_timeStep
        self.dt = torch.tensor([firstTimeStep], dtype=tensorType, device=device)
        self.t = torch.tensor([t], dtype=tensorType, device=device)
        self._export_n = export_n
        self._maxTimeStep = torch.tensor([60.0], dtype=tensorType, device=device)
        self._outpath = "outpath"
        self._export_enabled = True
        self._given_depth = torch.tensor([[0.0, 0.0]], dtype=tensorType, device=device)
        self._given_wl = torch.tensor([[0.0, 0.0]], dtype=tensorType, device=device)
        self._given_discharge = torch.tensor([[0.0, 0.0, 0.0]], dtype=tensorType, device=device)
        self.totalRain = torch.tensor([0.0], dtype=tensorType, device=device)
        self._rainfall_station_time_index = 0
        self._rainStationData = None

    # ------------------------------------------------------------------ setup
    def init__fluidField_tensor(self, mask, h, qx, qy, wl, z, device):
        """Compact the raster fields and build the neighbour table (HP/SWE_CUDA.py:115-227)."""
        mask = torch.as_tensor(mask, device=device)
        valid = mask > 0
        tt = self._tensorType
        self._landuseMask = torch.zeros(int(valid.sum()), dtype=torch.uint8, device=device)
        self._h_internal = torch.as_tensor(h, device=device)[valid].to(tt).contiguous()
        self._qx_internal = torch.as_tensor(qx, device=device)[valid].to(tt).contiguous()
        self._qy_internal = torch.as_tensor(qy, device=device)[valid].to(tt).contiguous()
        self._wl_internal = torch.as_tensor(wl, device=device)[valid].to(tt).contiguous()
        self._z_internal = torch.as_tensor(z, device=device)[valid].to(tt).contiguous()
        self._h_max = self._h_internal.clone()
        self._h_update = torch.zeros_like(self._h_internal)
        self._qx_update = torch.zeros_like(self._h_internal)
        self._qy_update = torch.zeros_like(self._h_internal)
        self._z_update = torch.zeros_like(self._h_internal)
        self._wetMask = torch.flatten((self._h_internal > 1.0e-6).nonzero()).to(torch.int32)
        self._normal = torch.tensor([[1.0, 0.0], [0.0, 1.0], [-1.0, 0.0], [0.0, -1.0]],
                                    dtype=tt, device=device)
        self._index = compact_index(mask)

    def set_boundary_tensor(self, boundList, device):
        for key, attr in (("H_GIVEN", "_given_depth"), ("WL_GIVEN", "_given_wl"),
                          ("Q_GIVEN", "_given_discharge")):
            if key in boundList:
                v = boundList[key]
                if isinstance(v, str):
                    v = np.loadtxt(v)
                setattr(self, attr, torch.as_tensor(np.asarray(v) if not torch.is_tensor(v) else v,
                                                    device=device).to(self._tensorType).contiguous())

    def set_landuse(self, mask, landuseMask, device):
        mask = torch.as_tensor(mask, device=device)
        self._landuseMask = torch.as_tensor(landuseMask, device=device)[mask > 0].to(
            torch.uint8).contiguous()

    set_landuse_cpu_to_gpu = set_landuse

    def set__frictionField_tensor(self, manning, device):
        if torch.is_tensor(manning):
            self._manning = manning.to(device=device, dtype=self._tensorType).contiguous()
        else:
            self._manning = torch.tensor([manning], dtype=self._tensorType, device=device)

    def set__infiltrationField_tensor(self, hydraulic_conductivity, capillary_head,
                                      water_content_diff, device):
        self._cumulativeWaterDepth = torch.zeros_like(self._h_internal)

        def as_t(v):
            if torch.is_tensor(v):
                return v.to(device=device, dtype=self._tensorType).contiguous()
            return torch.tensor([v], dtype=self._tensorType, device=device)

        self._hydraulic_conductivity = as_t(hydraulic_conductivity)
        self._capillary_head = as_t(capillary_head)
        self._water_content_diff = as_t(water_content_diff)

    def set_distributed_rainfall_station_Mask(self, mask, rainfall_station_Mask, device):
        mask = torch.as_tensor(mask, device=device)
        self._rainfall_station_Mask = torch.as_tensor(rainfall_station_Mask, device=device)[
            mask > 0].to(torch.int16).contiguous()
        self._rainfall_station_time_index = 0

    set_distributed_rainfall_station_Mask_cpu_to_gpu = set_distributed_rainfall_station_Mask

    def set_uniform_rainfall_time_index(self):
        self._rainfall_station_time_index = 0

    def setOutPutPath(self, outpath):
        self._outpath = outpath

    # ------------------------------------------------------------------ step
    def addFlux(self):
        """fluxMask -> active list -> HLLC flux accumulation (HP/SWE_CUDA.py:339-424)."""
        fm = torch.zeros_like(self._h_internal, dtype=torch.bool)
        self._ops.flux_mask(fm, self._h_internal, self._index, self.t)
        self._wetMask = torch.flatten(fm.nonzero()).to(torch.int32)
        op = self._ops.flux_2nd_order if self._secondOrder else self._ops.flux_1st_order
        op(self._wetMask, self._h_update, self._qx_update, self._qy_update, self._h_internal,
           self._wl_internal, self._z_internal, self._qx_internal, self._qy_internal,
           self._index, self._normal, self._given_depth, self._given_wl,
           self._given_discharge, self.dx, self.t, self.dt)

    def addInfiltrationSource(self):
        self._ops.infiltration(self._wetMask, self._h_update, self._landuseMask,
                               self._h_internal, self._hydraulic_conductivity,
                               self._capillary_head, self._water_content_diff,
                               self._cumulativeWaterDepth, self.dt)

    def _interp_rain(self, R: np.ndarray) -> np.ndarray:
        """Rain rates at t with the monotone row cursor (HP/SWE_CUDA.py:472-495)."""
        t = float(self.t.item())
        if t < R[-1, 0]:
            while not t < R[self._rainfall_station_time_index + 1, 0]:
                self._rainfall_station_time_index += 1
            k = self._rainfall_station_time_index
            per = (t - R[k, 0]) / (R[k + 1, 0] - R[k, 0])
            return R[k, 1:] + per * (R[k + 1, 1:] - R[k, 1:])
        return np.zeros(R.shape[1] - 1)

    def addStation_PrecipitationSource(self, rainfall_ndarray_data, device):
        rates = self._interp_rain(np.asarray(rainfall_ndarray_data, dtype=np.float64))
        self._rainStationData = torch.as_tensor(rates, dtype=self._tensorType, device=device)
        self._ops.station_rain(self._h_update, self._rainfall_station_Mask,
                               self._rainStationData, self.dt)

    def add_uniform_PrecipitationSource(self, rainfall_ndarray_data, device):
        rates = self._interp_rain(np.asarray(rainfall_ndarray_data, dtype=np.float64))
        self._rainStationData = torch.as_tensor(rates[:1], dtype=self._tensorType, device=device)
        self._h_update += self._rainStationData * self.dt

    def addRadarRainfall(self, rainfall_raster):
        self._h_update += rainfall_raster * self.dt

    def _update_list(self) -> torch.Tensor:
        return torch.flatten(((self._h_update.abs() > 0.0) | (self._h_internal >= 0.0))
                             .nonzero()).to(torch.int32)

    def friction_euler_update_cuda(self):
        self._wetMask = self._update_list()
        self._ops.friction_update(self._wetMask, self._h_update, self._qx_update,
                                  self._qy_update, self._z_update, self._landuseMask,
                                  self._h_internal, self._wl_internal, self._qx_internal,
                                  self._qy_internal, self._z_internal, self._manning, self.dt)

    def _advance_dt(self, time_upper: torch.Tensor, listed: int) -> None:
        """min -> 10x cap -> export clip -> t += dt (HP/SWE_CUDA.py:818-831)."""
        if listed != 0:
            self.dt = self._ops.device_min(self._accelerator_dt)
        self.dt = torch.where(time_upper < self.dt, time_upper, self.dt)
        nxt = float(self._export_n + 1) * self.export_timeStep
        if (self.dt + self.t).item() >= nxt:
            self.dt = nxt - self.t
            self.exportField()
            self._export_n += 1
        self.t += self.dt

    def time_friction_euler_update_cuda(self, device):
        time_upper = self.dt * 10.0
        self.friction_euler_update_cuda()
        self._accelerator_dt = torch.full(self._wetMask.size(), self._maxTimeStep.item(),
                                          dtype=self._tensorType, device=device)
        self._ops.update_timestep(self._wetMask, self._accelerator_dt, self._h_max,
                                  self._h_internal, self._qx_internal, self._qy_internal,
                                  self.dx, self.cfl, self.t, self.dt)
        self._advance_dt(time_upper, self._accelerator_dt.size(0))

    def euler_update(self):
        self._wetMask = torch.flatten(((self._h_update.abs() > 0.0) |
                                       (self._h_internal > 1.0e-6)).nonzero()).to(torch.int32)
        self._ops.euler_update(self._wetMask, self._h_update, self._qx_update,
                               self._qy_update, self._z_update, self._h_internal,
                               self._wl_internal, self._z_internal, self._qx_internal,
                               self._qy_internal)
        self._h_update.zero_()
        self._qx_update.zero_()
        self._qy_update.zero_()
        self._z_update.zero_()

    def time_update_cuda(self, device):
        time_upper = self.dt * 10.0
        self._wetMask = torch.flatten((self._h_internal > 1.0e-6).nonzero()).to(torch.int32)
        self._accelerator_dt = torch.full(self._wetMask.size(), self._maxTimeStep.item(),
                                          dtype=self._tensorType, device=device)
        self._ops.update_timestep(self._wetMask, self._accelerator_dt, self._h_max,
                                  self._h_internal, self._qx_internal, self._qy_internal,
                                  self.dx, self.cfl, self.t, self.dt)
        self._advance_dt(time_upper, self._accelerator_dt.size(0))

    def rungeKutta_update(self, rainfallMatrix, device):
        """Average of two Euler stages (HP/SWE_CUDA.py:870-892)."""
        h0, qx0, qy0 = (self._h_internal.clone(), self._qx_internal.clone(),
                        self._qy_internal.clone())
        for _ in range(2):
            self.addFlux()
            self.add_uniform_PrecipitationSource(rainfallMatrix, device)
            self.friction_euler_update_cuda()
        self._h_internal[:] = (self._h_internal + h0) / 2.0
        self._qx_internal[:] = (self._qx_internal + qx0) / 2.0
        self._qy_internal[:] = (self._qy_internal + qy0) / 2.0
        self._wl_internal[:] = self._h_internal + self._z_internal

    def run_updating(self, device):
        raise NotImplementedError(
            "run_updating uses the explicit friction op (frictionCalculation), which is "
            "outside the B200 hot path")

    # ------------------------------------------------------------------ output
    def exportField(self):
        """Save h, qx, qy, wl, h_max as <field>_<t>.pt (HP/SWE_CUDA.py:836-868)."""
        if not self._export_enabled:
            return
        os.makedirs(self._outpath, exist_ok=True)
        tag = str(self.t + self.dt)
        for name, x in (("h", self._h_internal), ("qx", self._qx_internal),
                        ("qy", self._qy_internal), ("wl", self._wl_internal),
                        ("h_max", self._h_max)):
            torch.save(x, os.path.join(self._outpath, f"{name}_{tag}.pt"))

    def observeGauges_write(self, observe_index, dataStoreList, n):
        if n % 10 == 0:
            row = [self.t.item()] + list(self._h_internal[observe_index].cpu().numpy())
            dataStoreList.append(row)

    def get_h(self):
        return self._h_internal

    def get_qx(self):
        return self._qx_internal

    def get_qy(self):
        return self._qy_internal
