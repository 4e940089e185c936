"""Tensor-level ops over libhipims_b200's C ABI.

Each function keeps the reference extension's positional signature, argument
meaning and in-place semantics (paths relative to CHANS-HiPIMS/hipims/cuda):

  flux_2nd_order      fluxCal_2ndOrder_jh_improved.cpp:28-53
  flux_1st_order      fluxCal_jh_modified_surface.cpp:28-53
  friction_update     friction_implicit_andUpdate_jh_interface.cpp:29-53
  update_timestep     timeControl.cpp:27-41
  station_rain        stationPrecipitation_interface.cpp:26-38
  flux_mask           fluxMaskGenerator.cpp:22-29
  euler_update        euler_update.cpp:27-44
  infiltration        infiltration_interface.cpp

Checks mirror the reference's CHECK_INPUT (``RuntimeError: <name> must be a
CUDA tensor.`` / ``... must be contiguous.``); in addition index/mask dtypes
are checked and CUDA launch errors raise instead of being printed.
"""
from __future__ import annotations

import threading

import torch

from . import _lib

_FLOAT_DTYPES = {torch.float32: _lib.HB_F32, torch.float64: _lib.HB_F64}


def _check_input(name: str, x: torch.Tensor) -> None:
    if not isinstance(x, torch.Tensor) or not x.is_cuda:
        raise RuntimeError(f"{name} must be a CUDA tensor. ")
    if not x.is_contiguous():
        raise RuntimeError(f"{name} must be contiguous. ")


def _check(named: dict) -> None:
    for k, v in named.items():
        _check_input(k, v)


def _dtype_of(h: torch.Tensor, others: dict) -> int:
    if h.dtype not in _FLOAT_DTYPES:
        raise RuntimeError(f"unsupported dtype {h.dtype}: expected float32 or float64")
    for k, v in others.items():
        if v.dtype != h.dtype:
            raise RuntimeError(f"{k} has dtype {v.dtype}, expected {h.dtype}")
    return _FLOAT_DTYPES[h.dtype]


def _need(name: str, x: torch.Tensor, dtype: torch.dtype) -> None:
    if x.dtype != dtype:
        raise RuntimeError(f"{name} must be {dtype} (got {x.dtype})")


def _p(x: torch.Tensor) -> int:
    return x.data_ptr()


def _stream(x: torch.Tensor) -> int:
    return torch.cuda.current_stream(x.device).cuda_stream


def _table(x: torch.Tensor) -> tuple[int, int]:
    if x.dim() == 1:
        return 1, x.shape[0]
    if x.dim() != 2:
        raise RuntimeError("boundary tables must be 1-D or 2-D")
    return x.shape[0], x.shape[1]


def _flux(order: int, wetMask, h_flux, qx_flux, qy_flux, h, wl, z, qx, qy, index, normal,
          given_depth, given_wl, given_q, dx, t, dt) -> None:
    _check(dict(h=h, wetMask=wetMask, wl=wl, z=z, qx=qx, qy=qy, index=index, dx=dx,
                normal=normal, given_q=given_q, given_wl=given_wl, given_depth=given_depth,
                dt=dt, t=t))
    dtype = _dtype_of(h, dict(h_flux=h_flux, qx_flux=qx_flux, qy_flux=qy_flux, wl=wl, z=z,
                              qx=qx, qy=qy, normal=normal, given_depth=given_depth,
                              given_wl=given_wl, given_q=given_q, dx=dx, t=t, dt=dt))
    _need("wetMask", wetMask, torch.int32)
    _need("index", index, torch.int32)
    M, N = wetMask.numel(), h.numel()
    if index.numel() != 5 * N:
        raise RuntimeError(f"index must hold 5*N = {5 * N} entries (got {index.numel()})")
    dr, dc = _table(given_depth)
    wr, wc = _table(given_wl)
    qr, qc = _table(given_q)
    L = _lib.lib()
    with torch.cuda.device(h.device):
        rc = L.hb_flux(order, dtype, M, N, _p(wetMask), _p(h_flux), _p(qx_flux), _p(qy_flux),
                       _p(h), _p(wl), _p(z), _p(qx), _p(qy), _p(index), _p(normal),
                       _p(given_depth), dr, dc, _p(given_wl), wr, wc, _p(given_q), qr, qc,
                       _p(dx), _p(t), _p(dt), _stream(h))
    _lib.check(rc, "addFlux")


def flux_2nd_order(wetMask, h_flux, qx_flux, qy_flux, h, wl, z, qx, qy, index, normal,
                   given_depth, given_wl, given_q, dx, t, dt) -> None:
    """fluxCal_2ndOrder_jh_improved.addFlux: MUSCL + hydrostatic + HLLC."""
    _flux(2, wetMask, h_flux, qx_flux, qy_flux, h, wl, z, qx, qy, index, normal,
          given_depth, given_wl, given_q, dx, t, dt)


def flux_1st_order(wetMask, h_flux, qx_flux, qy_flux, h, wl, z, qx, qy, index, normal,
                   given_depth, given_wl, given_q, dx, t, dt) -> None:
    """fluxCalculation_jh_modified_surface.addFlux: bed-only minmod + HLLC."""
    _flux(1, wetMask, h_flux, qx_flux, qy_flux, h, wl, z, qx, qy, index, normal,
          given_depth, given_wl, given_q, dx, t, dt)


def friction_update(wetMask, h_update, qx_update, qy_update, z_update, landuse, h, wl, qx,
                    qy, z, manning, dt) -> None:
    """friction_implicit_andUpdate_jh.addFriction_eulerUpdate."""
    _check(dict(wetMask=wetMask, landuse=landuse, h=h, qx=qx, z=z, wl=wl, qy=qy,
                h_update=h_update, z_update=z_update, qx_update=qx_update,
                qy_update=qy_update, dt=dt, manning=manning))
    dtype = _dtype_of(h, dict(h_update=h_update, qx_update=qx_update, qy_update=qy_update,
                              z_update=z_update, wl=wl, qx=qx, qy=qy, z=z, manning=manning,
                              dt=dt))
    _need("wetMask", wetMask, torch.int32)
    _need("landuse", landuse, torch.uint8)
    L = _lib.lib()
    with torch.cuda.device(h.device):
        rc = L.hb_friction_update(dtype, wetMask.numel(), _p(wetMask), _p(h_update),
                                  _p(qx_update), _p(qy_update), _p(z_update), _p(landuse),
                                  _p(h), _p(wl), _p(qx), _p(qy), _p(z), _p(manning), _p(dt),
                                  _stream(h))
    _lib.check(rc, "addFriction_eulerUpdate")


def update_timestep(wetMask, accelerator, h_max, h, qx, qy, dx, CFL, t, dt) -> None:
    """timeControl.updateTimestep: per-cell CFL step into `accelerator`, h_max."""
    _check(dict(wetMask=wetMask, h=h, h_max=h_max, qx=qx, qy=qy, dx=dx, CFL=CFL, dt=dt,
                t=t))
    dtype = _dtype_of(h, dict(accelerator=accelerator, h_max=h_max, qx=qx, qy=qy, dx=dx,
                              CFL=CFL))
    _need("wetMask", wetMask, torch.int32)
    if accelerator.numel() < wetMask.numel():
        raise RuntimeError("accelerator must hold one entry per listed cell")
    L = _lib.lib()
    with torch.cuda.device(h.device):
        rc = L.hb_timestep(dtype, wetMask.numel(), _p(wetMask), _p(accelerator), _p(h_max),
                           _p(h), _p(qx), _p(qy), _p(dx), _p(CFL), _p(t), _p(dt), _stream(h))
    _lib.check(rc, "updateTimestep")


def station_rain(h_update, rainStationMask, rainStationData, dt) -> None:
    """station_PrecipitationCalculation.addStation_Precipitation."""
    _check(dict(h_update=h_update, dt=dt, rainStationMask=rainStationMask,
                rainStationData=rainStationData))
    dtype = _dtype_of(h_update, dict(rainStationData=rainStationData, dt=dt))
    _need("rainStationMask", rainStationMask, torch.int16)
    L = _lib.lib()
    with torch.cuda.device(h_update.device):
        rc = L.hb_rain_station(dtype, rainStationMask.numel(), _p(h_update),
                               _p(rainStationMask), _p(rainStationData), _p(dt),
                               _stream(h_update))
    _lib.check(rc, "addStation_Precipitation")


def flux_mask(fluxMask, h, index, t) -> None:
    """fluxMask.update: fluxMask[i] = cell i or a neighbour (id > 0) is wet, or t == 0."""
    _check(dict(fluxMask=fluxMask, h=h, index=index, t=t))
    dtype = _dtype_of(h, dict(t=t))
    if fluxMask.dtype not in (torch.bool, torch.uint8):
        raise RuntimeError("fluxMask must be bool")
    _need("index", index, torch.int32)
    L = _lib.lib()
    with torch.cuda.device(h.device):
        rc = L.hb_flux_mask(dtype, h.numel(), _p(fluxMask), _p(h), _p(index), _p(t),
                            _stream(h))
    _lib.check(rc, "fluxMask.update")


def euler_update(updateMask, h_update, qx_update, qy_update, z_update, h, wl, z, qx,
                 qy) -> None:
    """euler_update.update: frictionless update of the listed cells."""
    _check(dict(updateMask=updateMask, h=h, qx=qx, qy=qy, wl=wl, z=z, qx_update=qx_update,
                qy_update=qy_update, h_update=h_update, z_update=z_update))
    dtype = _dtype_of(h, dict(h_update=h_update, qx_update=qx_update, qy_update=qy_update,
                              z_update=z_update, wl=wl, z=z, qx=qx, qy=qy))
    _need("updateMask", updateMask, torch.int32)
    L = _lib.lib()
    with torch.cuda.device(h.device):
        rc = L.hb_euler_update(dtype, updateMask.numel(), _p(updateMask), _p(h_update),
                               _p(qx_update), _p(qy_update), _p(z_update), _p(h), _p(wl),
                               _p(z), _p(qx), _p(qy), _stream(h))
    _lib.check(rc, "euler_update.update")


def infiltration(wetMask, h_update, landuse, h, hydraulic_conductivity, capillary_head,
                 water_content_diff, cumulative_depth, dt) -> None:
    """infiltrationCalculation.addinfiltration: Green-Ampt loss into h_update."""
    _check(dict(wetMask=wetMask, h_update=h_update, landuse=landuse, h=h,
                hydraulic_conductivity=hydraulic_conductivity, capillary_head=capillary_head,
                water_content_diff=water_content_diff, cumulative_depth=cumulative_depth,
                dt=dt))
    dtype = _dtype_of(h, dict(h_update=h_update, hydraulic_conductivity=hydraulic_conductivity,
                              capillary_head=capillary_head,
                              water_content_diff=water_content_diff,
                              cumulative_depth=cumulative_depth, dt=dt))
    _need("wetMask", wetMask, torch.int32)
    _need("landuse", landuse, torch.uint8)
    L = _lib.lib()
    with torch.cuda.device(h.device):
        rc = L.hb_infiltration(dtype, wetMask.numel(), _p(wetMask), _p(h_update), _p(landuse),
                               _p(h), _p(hydraulic_conductivity), _p(capillary_head),
                               _p(water_content_diff), _p(cumulative_depth), _p(dt),
                               _stream(h))
    _lib.check(rc, "addinfiltration")


# hb_min_reduce workspaces, one per (device, stream), grown on demand: the
# kernel leaves its block counter at zero after every call, so a workspace is
# zero-filled once, when it is allocated, and calls ordered on one stream can
# share it.
_MIN_WS: dict = {}
_MIN_WS_LOCK = threading.Lock()


def _min_workspace(x: torch.Tensor, nbytes: int) -> torch.Tensor:
    key = (x.device.index, _stream(x))
    with _MIN_WS_LOCK:
        ws = _MIN_WS.get(key)
        if ws is None or ws.numel() < nbytes:
            ws = torch.zeros(nbytes, dtype=torch.uint8, device=x.device)
            _MIN_WS[key] = ws
        return ws


def device_min(x: torch.Tensor, out: torch.Tensor | None = None) -> torch.Tensor:
    """min(x) on the device without a host sync (replaces torch.min(accelerator)).
    Allocates nothing per call once its per-stream workspace has grown to the
    largest size seen."""
    _check_input("x", x)
    dtype = _dtype_of(x, {})
    if out is None:
        out = torch.empty(1, dtype=x.dtype, device=x.device)
    L = _lib.lib()
    nbytes = L.hb_min_reduce_workspace_size(x.numel())
    ws = _min_workspace(x, nbytes) if nbytes else None
    with torch.cuda.device(x.device):
        rc = L.hb_min_reduce(dtype, x.numel(), _p(x), _p(out), _p(ws) if ws is not None else None,
                             _stream(x))
    _lib.check(rc, "device_min")
    return out


def gather(cell_offsets: torch.Tensor, h: torch.Tensor, qx: torch.Tensor | None = None,
           qy: torch.Tensor | None = None, velocities: bool = False):
    """Depth (and u = qx/h, v = qy/h, 0 when dry) at flat element offsets."""
    _check(dict(cell_offsets=cell_offsets, h=h))
    _need("cell_offsets", cell_offsets, torch.int64)
    dtype = _dtype_of(h, {})
    n = cell_offsets.numel()
    oh = torch.empty(n, dtype=h.dtype, device=h.device)
    ou = ov = None
    if velocities:
        if qx is None or qy is None:
            raise RuntimeError("velocities need qx and qy")
        ou = torch.empty_like(oh)
        ov = torch.empty_like(oh)
    L = _lib.lib()
    with torch.cuda.device(h.device):
        rc = L.hb_gather(dtype, n, _p(cell_offsets), _p(h),
                         _p(qx) if qx is not None else None, _p(qy) if qy is not None else None,
                         _p(oh), _p(ou) if ou is not None else None,
                         _p(ov) if ov is not None else None, _stream(h))
    _lib.check(rc, "gather")
    return (oh, ou, ov) if velocities else oh
