"""FusedSolver: dense-tile, one-kernel-per-step HiPIMS solver (single or batched).

A catchment is given as rasters (type-code mask, z, h, qx, qy, Manning zone)
exactly as the reference's ``Godunov.init__fluidField_tensor`` takes them; the
solver keeps them dense (no compaction, no neighbour table) in the padded
layout of include/hipims_b200_fused.h and advances every instance of a batch
with one ``hb_fused_step`` launch per step.  ``t`` and ``dt`` live in a device
control block per instance, so K steps can be enqueued (or replayed from a
CUDA graph) without a host sync.

Semantics follow the reference step (HP/SWE_CUDA.py:339-424, 497-502,
780-831): the same activity mask, MUSCL/hydrostatic/HLLC fluxes, bed slope,
rain, implicit friction, CFL step with the 10x growth cap and the clip to
export times.
"""
from __future__ import annotations

import ctypes
import dataclasses
import math
import os
from typing import Sequence

import numpy as np
import torch

from . import _lib
from .topology import decode_bc


@dataclasses.dataclass
class Catchment:
    """One instance.  Rasters are [rows, cols]; mask > 0 marks valid cells and
    holds the reference type code (1 interior, e.g. 50 = OPEN id 0)."""

    mask: np.ndarray
    z: np.ndarray
    h: np.ndarray
    qx: np.ndarray | None = None
    qy: np.ndarray | None = None
    zone: np.ndarray | None = None          # Manning zone per cell (< 16)
    manning: Sequence[float] = (0.03,)
    dx: float = 1.0
    cfl: float = 0.5
    t0: float = 0.0
    dt0: float = 1.0e-4
    export_step: float = 0.0                # 0: no export clipping
    t_end: float = math.inf
    halt_on_export: bool = False
    rain: np.ndarray | None = None          # [T, 2] time (s), rate (m/s)
    rain_mult: float = 1.0
    given_depth: np.ndarray | None = None   # [Td, 1 + nH]
    given_wl: np.ndarray | None = None      # [Tw, 1 + nW]
    given_q: np.ndarray | None = None       # [Tq, 1 + 2 nQ]
    h_max: np.ndarray | None = None         # default: h
    dt_replay: np.ndarray | None = None     # frozen schedule: dt of step k+1 = dt_replay[k]
    # Green-Ampt infiltration: {"ks", "psi", "dtheta"} per Manning zone (m/s, m, -)
    infiltration: dict | None = None
    cum: np.ndarray | None = None           # initial cumulative infiltrated depth (m)
    # station rain: station id of every cell (raster); rain is then [T, 1 + S]
    # with one rate column per station (HP/SWE_CUDA.py:472-502)
    rain_station: np.ndarray | None = None


def block_datum(valid: np.ndarray, z: np.ndarray, block: int = 64) -> np.ndarray:
    """Integer bed datum of every block x block block: floor of the lowest
    valid bed elevation in it (0 for a block without valid cells)."""
    rows, cols = valid.shape
    nby, nbx = (rows + block - 1) // block, (cols + block - 1) // block
    zv = np.full((nby * block, nbx * block), np.inf)
    zv[:rows, :cols] = np.where(valid, z, np.inf)
    m = zv.reshape(nby, block, nbx, block).min(axis=(1, 3))
    return np.where(np.isfinite(m), np.floor(np.where(np.isfinite(m), m, 0.0)), 0.0)


def _round_up(x: int, m: int) -> int:
    return (x + m - 1) // m * m


# Reach of a tile's stencil as the tile classification counts it: rows above
# and below, columns left and right (the staged box of the step kernel).
_REACH_Y, _REACH_X = 2, 4


def tile_grid_cost(valid: np.ndarray, tile: tuple[int, int], origin: tuple[int, int],
                   bug: tuple[int, int] | None = None) -> float:
    """Modelled time of one step of the two-cells-per-lane kernel over
    `valid` when `origin` = (rows, cols) of no-data are put above and left of
    the raster, in units of an all-valid tile: a general tile costs
    0.4 + 1.1 x (rows per warp) / (ty / 4), its four warps sharing the rows
    from its first to its last row with a valid cell; a tile without valid
    cells 0.1."""
    valid = np.asarray(valid, dtype=bool)
    S = _prefix(valid)
    return float(_grid_cost(S, valid.shape, tile, np.array([origin[0]]), np.array([origin[1]]),
                            bug)[0])


def _prefix(valid: np.ndarray) -> np.ndarray:
    rows, cols = valid.shape
    S = np.zeros((rows + 1, cols + 1), dtype=np.int32)
    S[1:, 1:] = np.cumsum(np.cumsum(valid, axis=0, dtype=np.int32), axis=1)
    return S


def _grid_cost(S, shape, tile, sy: np.ndarray, sx: np.ndarray, bug) -> np.ndarray:
    """tile_grid_cost for origins (sy[k], sx[k]) at once (prefix sums S)."""
    rows, cols = shape
    ty, tx = tile

    def count(y0, y1, x0, x1):  # valid cells in [y0, y1) x [x0, x1), clipped
        y0, y1 = np.clip(y0, 0, rows), np.clip(y1, 0, rows)
        x0, x1 = np.clip(x0, 0, cols), np.clip(x1, 0, cols)
        return S[y1, x1] - S[y0, x1] - S[y1, x0] + S[y0, x0]

    nty, ntx = (rows + sy + ty - 1) // ty, (cols + sx + tx - 1) // tx  # per origin
    y0 = np.arange(nty.max())[None, :, None] * ty - sy[:, None, None]
    x0 = np.arange(ntx.max())[None, None, :] * tx - sx[:, None, None]
    exists = ((np.arange(nty.max())[None, :, None] < nty[:, None, None]) &
              (np.arange(ntx.max())[None, None, :] < ntx[:, None, None]))
    by0, by1 = y0 - _REACH_Y, y0 + ty + _REACH_Y
    bx0, bx1 = x0 - _REACH_X, x0 + tx + _REACH_X
    inside = (by0 >= 0) & (by1 <= rows) & (bx0 >= 0) & (bx1 <= cols)
    allv = inside & (count(by0, by1, bx0, bx1) == (by1 - by0) * (bx1 - bx0))
    if bug is not None and bug[0] >= 0:
        allv &= ~((bug[0] >= by0) & (bug[0] < by1) & (bug[1] >= bx0) & (bug[1] < bx1))
    cost = np.where(allv & exists, 1.0, 0.0)
    g = np.nonzero(exists & ~allv)  # general tiles: rows from the first to the last live one
    gy = np.broadcast_to(y0, allv.shape)[g][:, None] + np.arange(ty)[None, :]
    gx = np.broadcast_to(x0, allv.shape)[g][:, None]
    live = count(gy, gy + 1, gx, gx + tx) > 0
    lo = np.where(live.any(-1), live.argmax(-1), 0)
    hi = np.where(live.any(-1), ty - live[:, ::-1].argmax(-1), 0)
    per_warp = -(-(hi - lo) // 4)  # rows of the warp that walks most
    cost[g] = np.where(hi > lo, 0.4 + 1.1 * per_warp / (ty / 4), 0.1)
    return cost.sum(axis=(1, 2))


def tile_origin(valid: np.ndarray, tile: tuple[int, int],
                bug: tuple[int, int] | None = None) -> tuple[int, int]:
    """Rows and columns of no-data to put above and left of a catchment so
    that its tile grid costs least under tile_grid_cost: the all-valid tiles
    then start where the valid cells do, and the tiles over the catchment's
    edges hold as few rows as they can.  Coordinate descent over the column
    and row shifts (smallest shift among equals)."""
    ty, tx = tile
    valid = np.asarray(valid, dtype=bool)
    if not valid.any():
        return (0, 0)
    S = _prefix(valid)
    sy, sx = 0, 0

    def best(cy, cx):
        k = int(np.argmin(_grid_cost(S, valid.shape, tile, cy, cx, bug)))  # first minimum
        return int(cy[k]), int(cx[k])

    for axis in (1, 0, 1):
        n = ty if axis == 0 else tx
        sy, sx = best(np.arange(n) if axis == 0 else np.full(n, sy),
                      np.arange(n) if axis == 1 else np.full(n, sx))
    return (sy, sx)


def _shift_catchment(c: Catchment, sy: int, sx: int) -> Catchment:
    """c with sy rows and sx columns of no-data (zeros) above and left of
    every raster field."""
    if sy == 0 and sx == 0:
        return c
    pad = lambda a: None if a is None else np.pad(np.asarray(a), ((sy, 0), (sx, 0)))
    return dataclasses.replace(
        c, mask=pad(c.mask), z=pad(c.z), h=pad(c.h), qx=pad(c.qx), qy=pad(c.qy),
        zone=pad(c.zone), h_max=pad(c.h_max), cum=pad(c.cum), rain_station=pad(c.rain_station))


def _first_valid_cell(mask) -> tuple[int, int] | None:
    """(row, col) of the first valid cell in row-major order (compacted
    cell 0 of the reference), or None."""
    m = np.asarray(mask)
    flat = np.flatnonzero(m.ravel() > 0)
    return None if flat.size == 0 else (int(flat[0] // m.shape[1]), int(flat[0] % m.shape[1]))


class _Instance:
    """Device arrays of one catchment in the padded dense layout.

    origin = (sy, sx): the kernels see the catchment with sy rows and sx
    columns of no-data above and left of it (the tile grid starts that far
    before the raster).  `raster()` views and `valid` are in the catchment's
    own coordinates; `rows`, `cols` and `bug` in the kernels' raster."""

    def __init__(self, c: Catchment, dtype: torch.dtype, device, tile: tuple[int, int],
                 origin: tuple[int, int] = (0, 0)):
        sy, sx = (int(origin[0]), int(origin[1]))
        if sy < 0 or sx < 0:
            raise ValueError("the tile grid origin must be >= 0 in rows and columns")
        self.origin = (sy, sx)
        self.crows, self.ccols = np.asarray(c.mask).shape
        c0 = c
        c = _shift_catchment(c, sy, sx)
        rows, cols = c.mask.shape
        self.rows, self.cols = rows, cols
        self.dx = float(c.dx)
        ty, tx = tile
        self.tiles_y = (rows + ty - 1) // ty
        self.tiles_x = (cols + tx - 1) // tx
        rows_s = _round_up(rows, 64) + 2 * _lib.HB_PAD_Y
        pitch = _round_up(_round_up(cols, 64) + 2 * _lib.HB_PAD_X, 32)
        code_pitch = _round_up(_round_up(cols, 64) + 2 * _lib.HB_CODE_PAD_X, 128)
        self.rows_s, self.pitch, self.code_pitch = rows_s, pitch, code_pitch
        PY, PX, CPX = _lib.HB_PAD_Y, _lib.HB_PAD_X, _lib.HB_CODE_PAD_X
        mask = np.asarray(c.mask)
        valid = mask > 0
        self.valid = valid[sy:, sx:]
        self.n_valid = int(valid.sum())

        # boundary classes: distinct type codes of valid cells
        codes = sorted(set(int(v) for v in np.unique(mask[valid])))
        if len(codes) > _lib.HB_MAX_CLASSES - 1:
            raise ValueError(f"at most {_lib.HB_MAX_CLASSES - 1} distinct cell codes per "
                             f"catchment in the fused path (got {len(codes)})")
        self.class_codes = codes
        cls_of = {code: k for k, code in enumerate(codes)}
        cls = np.full(mask.shape, _lib.HB_NODATA_CLASS, dtype=np.uint8)
        for code, k in cls_of.items():
            cls[mask == code] = k
        zone = np.zeros(mask.shape, dtype=np.uint8) if c.zone is None else np.asarray(c.zone)
        if zone.max(initial=0) >= _lib.HB_MAX_ZONES or len(c.manning) > _lib.HB_MAX_ZONES:
            raise ValueError(f"at most {_lib.HB_MAX_ZONES} Manning zones in the fused path")
        code_r = ((cls.astype(np.uint8) << 4) | (zone.astype(np.uint8) & 15)).astype(np.uint8)
        code_np = np.full((rows_s, code_pitch), _lib.HB_NODATA_CLASS << 4, dtype=np.uint8)
        code_np[PY:PY + rows, CPX:CPX + cols] = code_r

        # datum per 64 x 64 block (FP32 only)
        z = np.asarray(c.z, dtype=np.float64)
        fp32 = dtype == torch.float32
        nby, nbx = (rows + 63) // 64, (cols + 63) // 64
        datum = block_datum(valid, z) if fp32 else np.zeros((nby, nbx), dtype=np.float64)
        self.datum_np = datum
        dfull = np.repeat(np.repeat(datum, 64, axis=0), 64, axis=1)[:rows, :cols]
        zrel = np.where(valid, z - dfull, 0.0)

        def dense(a, fill=0.0):
            out = np.full((rows_s, pitch), fill, dtype=np.float64)
            if a is not None:
                out[PY:PY + rows, PX:PX + cols] = np.where(valid, np.asarray(a, np.float64), 0.0)
            return torch.as_tensor(out, dtype=dtype, device=device).contiguous()

        h = dense(c.h)
        qx = dense(c.qx)
        qy = dense(c.qy)
        self.initial = (h.clone(), qx.clone(), qy.clone())
        self.h = [h, h.clone()]
        self.qx = [qx, qx.clone()]
        self.qy = [qy, qy.clone()]
        self.z = dense(zrel)
        self.h_max = dense(c.h if c.h_max is None else c.h_max)
        self.initial_h_max = self.h_max.clone()
        self.code = torch.as_tensor(code_np, device=device).contiguous()
        self.datum = torch.as_tensor(datum, dtype=torch.float32, device=device).contiguous()
        self.z_abs_offset = dfull[sy:, sx:]

        def table(a, width):
            if a is None:
                a = np.zeros((1, width))
            a = np.atleast_2d(np.asarray(a, dtype=np.float64))
            return torch.as_tensor(a, device=device).contiguous()

        self.given_depth = table(c.given_depth, 2)
        self.given_wl = table(c.given_wl, 2)
        self.given_q = table(c.given_q, 3)
        self.rain = None if c.rain is None else table(c.rain, 2)
        self.dt_replay = None if c.dt_replay is None else torch.as_tensor(
            np.asarray(c.dt_replay, dtype=np.float64), device=device).contiguous()
        self.rain_station = None
        if c.rain_station is not None:
            st = np.where(valid, np.asarray(c.rain_station), 0).astype(np.int64)
            n_st = (self.rain.shape[1] - 1) if self.rain is not None else 0
            if n_st < 1 or st.min(initial=0) < 0 or st.max(initial=0) >= n_st:
                raise ValueError("rain_station ids must index the rain table's station columns")
            dense_st = np.zeros((rows_s, pitch), dtype=np.int16)
            dense_st[PY:PY + rows, PX:PX + cols] = st.astype(np.int16)
            self.rain_station = torch.as_tensor(dense_st, device=device).contiguous()
            self.station_cells = torch.as_tensor(
                np.bincount(st[valid], minlength=n_st).astype(np.float64), device=device)
            self.station_rate = torch.zeros(n_st, dtype=torch.float64, device=device)
        self.cum = None
        self.infil = None
        if c.infiltration is not None:
            self.cum = dense(c.cum)
            self.initial_cum = self.cum.clone()

            def per_zone(key):
                v = [float(x) for x in np.atleast_1d(c.infiltration[key])]
                if len(v) > _lib.HB_MAX_ZONES:
                    raise ValueError(f"at most {_lib.HB_MAX_ZONES} infiltration zones")
                return v + [0.0] * (_lib.HB_MAX_ZONES - len(v))

            self.infil = {k: per_zone(k) for k in ("ks", "psi", "dtheta")}

        # position of compacted cell 0 (fluxMask quirk)
        if self.n_valid:
            flat = int(np.flatnonzero(valid.ravel())[0])
            self.bug = (flat // cols, flat % cols)
        else:
            self.bug = (-1, -1)
        self.bc_type = [1] * _lib.HB_MAX_CLASSES
        self.bc_id = [0] * _lib.HB_MAX_CLASSES
        for code, k in cls_of.items():
            bt, bid = decode_bc(code)
            self.bc_type[k] = bt
            self.bc_id[k] = bid
        self.manning = list(c.manning) + [0.0] * (_lib.HB_MAX_ZONES - len(c.manning))
        self.catchment = c0

    def raster(self, t: torch.Tensor) -> torch.Tensor:
        """The catchment's rows x cols view of a dense array."""
        PY, PX = _lib.HB_PAD_Y + self.origin[0], _lib.HB_PAD_X + self.origin[1]
        return t[PY:PY + self.crows, PX:PX + self.ccols]


class FusedSolver:
    """Advance one or more catchments with the fused dense-tile kernel.

    order 2 (default): the reference's 2nd-order scheme (MUSCL, `secondOrder`
    True); order 1: its 1st-order scheme (`secondOrder` False, the coupled
    server's choice, CHANS-HiPIMS_server.py).

    tile = (rows, cols): (32, 64) runs two cells per lane (FP32, either order:
    the default there); (32, 32) and (64, 32) one cell per lane (every dtype
    and order).

    origin: rows and columns of no-data the kernels see above and left of each
    catchment, i.e. where the tile grid starts (results are given back in the
    catchment's own coordinates).  None: chosen per catchment by tile_origin
    for 32 x 64 tiles, (0, 0) for the others; a pair: every catchment; a list:
    one pair per catchment.  In FP32 the bed datum blocks move with the grid,
    so runs on different origins differ by round-off."""

    def __init__(self, catchments: Catchment | Sequence[Catchment], dtype=torch.float32,
                 tile: tuple[int, int] | None = None, device="cuda", grid_blocks: int = 0,
                 exact_fp32: bool = False, kernel: str = "rows", minb: int = 0,
                 order: int = 2, origin=None):
        if isinstance(catchments, Catchment):
            catchments = [catchments]
        if dtype not in (torch.float32, torch.float64):
            raise ValueError("dtype must be float32 or float64")
        if order not in (1, 2):
            raise ValueError("order must be 1 or 2")
        if order == 1 and kernel != "rows":
            raise ValueError("the 1st-order scheme runs in the rows kernel")
        self.device = torch.device(device)
        self.dtype = dtype
        self.order = order
        if tile is None:
            # FP32 (not exact_fp32): 32 x 64 tiles, two cells per lane;
            # otherwise the 32 x 32 row-walking tiles
            pairs = dtype == torch.float32 and kernel == "rows" and not exact_fp32
            tile = (32, 64) if pairs else (32, 32)
        self.tile = tuple(tile)
        if origin is None:
            origins = [tile_origin(np.asarray(c.mask) > 0, self.tile, _first_valid_cell(c.mask))
                       if self.tile == (32, 64) else (0, 0) for c in catchments]
        elif len(origin) == 2 and np.isscalar(origin[0]):
            origins = [tuple(origin)] * len(catchments)
        else:
            origins = [tuple(o) for o in origin]
            if len(origins) != len(catchments):
                raise ValueError("origin: one (rows, cols) pair per catchment")
        self.inst = [_Instance(c, dtype, self.device, self.tile, o)
                     for c, o in zip(catchments, origins)]
        n = len(self.inst)
        self._ctrl_size = ctypes.sizeof(_lib.HbCtrl)
        ctrl_host = (_lib.HbCtrl * n)()
        tile_inst = []
        begin = 0
        recs = (_lib.HbInstance * n)()
        self.ctrl = torch.zeros(n * self._ctrl_size, dtype=torch.uint8, device=self.device)
        for k, (ins, c) in enumerate(zip(self.inst, catchments)):
            cb = ctrl_host[k]
            cb.t, cb.dt = c.t0, c.dt0
            cb.export_step = c.export_step
            cb.t_end = c.t_end
            cb.rain_mult = c.rain_mult
            cb.halt_on_export = int(c.halt_on_export)
            r = recs[k]
            r.rows, r.cols = ins.rows, ins.cols
            r.tiles_x, r.tiles_y = ins.tiles_x, ins.tiles_y
            r.tile_begin = begin
            r.pitch, r.code_pitch = ins.pitch, ins.code_pitch
            r.datum_ny, r.datum_nx = ins.datum_np.shape
            r.bug_y, r.bug_x = ins.bug
            r.h[0], r.h[1] = ins.h[0].data_ptr(), ins.h[1].data_ptr()
            r.qx[0], r.qx[1] = ins.qx[0].data_ptr(), ins.qx[1].data_ptr()
            r.qy[0], r.qy[1] = ins.qy[0].data_ptr(), ins.qy[1].data_ptr()
            r.z = ins.z.data_ptr()
            r.h_max = ins.h_max.data_ptr()
            r.code = ins.code.data_ptr()
            r.datum = ins.datum.data_ptr() if dtype == torch.float32 else None
            r.ctrl = self.ctrl.data_ptr() + k * self._ctrl_size
            if ins.rain is not None:
                r.rain_tab = ins.rain.data_ptr()
                r.rain_rows, r.rain_cols = ins.rain.shape
            r.given_depth = ins.given_depth.data_ptr()
            r.depth_rows, r.depth_cols = ins.given_depth.shape
            r.given_wl = ins.given_wl.data_ptr()
            r.wl_rows, r.wl_cols = ins.given_wl.shape
            r.given_q = ins.given_q.data_ptr()
            r.q_rows, r.q_cols = ins.given_q.shape
            r.dx, r.cfl = c.dx, c.cfl
            for z_ in range(_lib.HB_MAX_ZONES):
                r.manning[z_] = ins.manning[z_]
            for q in range(_lib.HB_MAX_CLASSES):
                r.bc_type[q] = ins.bc_type[q]
                r.bc_id[q] = ins.bc_id[q]
            r.n_valid = ins.n_valid
            if ins.dt_replay is not None:
                r.dt_replay = ins.dt_replay.data_ptr()
                r.n_replay = ins.dt_replay.numel()
            if ins.rain_station is not None:
                if kernel == "tasks":
                    raise ValueError("station rain needs the rows kernel")
                r.rain_station = ins.rain_station.data_ptr()
                r.station_rate = ins.station_rate.data_ptr()
                r.station_cells = ins.station_cells.data_ptr()
                r.n_stations = ins.station_rate.numel()
            if ins.cum is not None:
                if kernel == "tasks":
                    raise ValueError("infiltration needs the rows kernel")
                r.cum = ins.cum.data_ptr()
                for z_ in range(_lib.HB_MAX_ZONES):
                    r.ks[z_] = ins.infil["ks"][z_]
                    r.psi[z_] = ins.infil["psi"][z_]
                    r.dtheta[z_] = ins.infil["dtheta"][z_]
            nt = ins.tiles_x * ins.tiles_y
            tile_inst.extend([k] * nt)
            begin += nt
        self.n_tiles = begin
        self._ctrl_init = bytes(ctrl_host)
        self.ctrl.copy_(torch.frombuffer(bytearray(ctrl_host), dtype=torch.uint8))
        self._recs_host = recs
        self.records = torch.frombuffer(bytearray(recs), dtype=torch.uint8).to(self.device)
        self.tile_instance = torch.tensor(tile_inst, dtype=torch.int32, device=self.device)
        b = _lib.HbFusedBatch()
        b.dtype = _lib.HB_F32 if dtype == torch.float32 else _lib.HB_F64
        b.n_instances = n
        b.n_tiles = self.n_tiles
        b.tile_y, b.tile_x = self.tile
        b.grid_blocks = grid_blocks
        b.order = order
        sources = any(i.cum is not None or i.rain_station is not None for i in self.inst)
        b.flags = ((1 if exact_fp32 else 0) | (2 if kernel == "tasks" else 0) |
                   (4 if sources else 0) | (minb << 8))
        b.instances_host = ctypes.addressof(self._recs_host)
        b.instances = self.records.data_ptr()
        b.tile_instance = self.tile_instance.data_ptr()
        L = _lib.lib()
        ws = L.hb_fused_workspace_size(ctypes.byref(b))
        self.workspace = torch.zeros(max(ws, 256), dtype=torch.uint8, device=self.device)
        b.workspace = self.workspace.data_ptr()
        self.batch = b
        self._graph = None
        self._graph_steps = 0
        self.prepare()

    # ----------------------------------------------------------------- control
    def record_ptr(self, k: int = 0) -> int:
        """Device address of instance k's hb_instance record."""
        return self.records.data_ptr() + k * ctypes.sizeof(_lib.HbInstance)

    def set_manning(self, k: int, manning: Sequence[float]) -> None:
        """Replace the Manning coefficients (per zone) of instance k."""
        if len(manning) > _lib.HB_MAX_ZONES:
            raise ValueError(f"at most {_lib.HB_MAX_ZONES} Manning zones")
        vals = [float(v) for v in manning] + [0.0] * (_lib.HB_MAX_ZONES - len(manning))
        self.inst[k].manning = vals
        for z_ in range(_lib.HB_MAX_ZONES):
            self._recs_host[k].manning[z_] = vals[z_]
        self.records.copy_(torch.frombuffer(bytearray(self._recs_host), dtype=torch.uint8))

    def set_external_dt(self, on: bool = True) -> None:
        """Defer the clock of every instance to hb_fused_finish (strips of one
        catchment: the next dt needs the wave speed of all strips)."""
        n = len(self.inst)
        init = (_lib.HbCtrl * n).from_buffer_copy(self._ctrl_init)
        cs = self.controls()
        for k in range(n):
            init[k].external_dt = cs[k].external_dt = 1 if on else 0
        self._ctrl_init = bytes(init)
        self.write_controls(cs)

    def reset(self, rain_mult: Sequence[float] | float | None = None) -> None:
        """Back to the initial state and control blocks of the catchments
        (t0, dt0, step 0), optionally with new rain multipliers; re-prepares."""
        n = len(self.inst)
        arr = (_lib.HbCtrl * n).from_buffer_copy(self._ctrl_init)
        if rain_mult is not None:
            mult = [rain_mult] * n if np.isscalar(rain_mult) else list(rain_mult)
            for k in range(n):
                arr[k].rain_mult = float(mult[k])
        for ins in self.inst:
            h0, qx0, qy0 = ins.initial
            for buf in range(2):
                ins.h[buf].copy_(h0)
                ins.qx[buf].copy_(qx0)
                ins.qy[buf].copy_(qy0)
            ins.h_max.copy_(ins.initial_h_max)
            if ins.cum is not None:
                ins.cum.copy_(ins.initial_cum)
        self.ctrl.copy_(torch.frombuffer(bytearray(arr), dtype=torch.uint8))
        self.prepare()

    def _stream(self) -> int:
        return torch.cuda.current_stream(self.device).cuda_stream

    def prepare(self) -> None:
        with torch.cuda.device(self.device):
            _lib.check(_lib.lib().hb_fused_prepare(ctypes.byref(self.batch), self._stream()),
                       "hb_fused_prepare")

    def step(self, nsteps: int = 1) -> None:
        """Enqueue nsteps fused steps (no host sync)."""
        with torch.cuda.device(self.device):
            _lib.check(_lib.lib().hb_fused_step(ctypes.byref(self.batch), int(nsteps),
                                                self._stream()), "hb_fused_step")

    def step_noalloc(self, nsteps: int = 1, prepare: bool = False) -> None:
        """Enqueue nsteps steps through hb_fused_step_noalloc, which keeps its
        scratch in the library's fixed device array instead of this solver's
        workspace (for hosts that cannot allocate device memory).  Pass
        prepare=True on the first such call."""
        with torch.cuda.device(self.device):
            _lib.check(_lib.lib().hb_fused_step_noalloc(ctypes.byref(self.batch), int(nsteps),
                                                        1 if prepare else 0, self._stream()),
                       "hb_fused_step_noalloc")

    def run_persistent(self, nsteps: int = 1, budget_cycles: int = 0) -> None:
        """Enqueue nsteps steps of every instance as ONE persistent cooperative
        launch (hb_fused_run; FP32 2nd order, 32 x 64 tiles): the same results
        as step(nsteps).  budget_cycles bounds every grid-barrier wait (0: the
        library's default, about a second); a wait that gives up sets status
        bit 8, which check() reports."""
        with torch.cuda.device(self.device):
            _lib.check(_lib.lib().hb_fused_run(ctypes.byref(self.batch), int(nsteps),
                                               int(budget_cycles), self._stream()),
                       "hb_fused_run")

    def capture_persistent(self, nsteps: int) -> None:
        """Capture one persistent launch of nsteps steps in a CUDA graph for
        replay()."""
        self._graph = None
        torch.cuda.synchronize(self.device)
        s = torch.cuda.Stream(self.device)
        s.wait_stream(torch.cuda.current_stream(self.device))
        g = torch.cuda.CUDAGraph()
        with torch.cuda.stream(s):
            with torch.cuda.graph(g, stream=s):
                _lib.check(_lib.lib().hb_fused_run(ctypes.byref(self.batch), int(nsteps), 0,
                                                   s.cuda_stream), "hb_fused_run")
        torch.cuda.current_stream(self.device).wait_stream(s)
        self._graph = g
        self._graph_steps = nsteps

    def capture(self, nsteps: int) -> None:
        """Capture nsteps steps in a CUDA graph for replay()."""
        self._graph = None
        torch.cuda.synchronize(self.device)
        s = torch.cuda.Stream(self.device)
        s.wait_stream(torch.cuda.current_stream(self.device))
        g = torch.cuda.CUDAGraph()
        with torch.cuda.stream(s):
            with torch.cuda.graph(g, stream=s):
                _lib.check(_lib.lib().hb_fused_step(ctypes.byref(self.batch), int(nsteps),
                                                    s.cuda_stream), "hb_fused_step")
        torch.cuda.current_stream(self.device).wait_stream(s)
        self._graph = g
        self._graph_steps = nsteps

    def replay(self) -> None:
        if self._graph is None:
            raise RuntimeError("capture() first")
        self._graph.replay()

    def controls(self) -> list[_lib.HbCtrl]:
        """Host copy of every instance's control block (syncs)."""
        raw = bytearray(self.ctrl.cpu().numpy().tobytes())
        n = len(self.inst)
        arr = (_lib.HbCtrl * n).from_buffer_copy(raw)
        return list(arr)

    def write_controls(self, ctrls: Sequence[_lib.HbCtrl]) -> None:
        n = len(self.inst)
        arr = (_lib.HbCtrl * n)(*ctrls)
        self.ctrl.copy_(torch.frombuffer(bytearray(arr), dtype=torch.uint8))

    STATUS = {1: "non-finite time step", 2: "a tile's data did not arrive in time",
              4: "non-finite depth",
              8: "a grid barrier of the persistent step gave up (budget exhausted)"}

    def check(self) -> None:
        """Raise if a step flagged a failure in any control block (syncs)."""
        bad = []
        for k, c in enumerate(self.controls()):
            if c.status:
                why = ", ".join(m for b, m in self.STATUS.items() if c.status & b)
                bad.append(f"instance {k} at t = {c.t:.6g} s, step {c.step}: {why}")
        if bad:
            raise FloatingPointError("fused step failed: " + "; ".join(bad))

    def resume(self, k: int | None = None) -> None:
        """Clear the halted flag (after an export halt) of one or all instances."""
        cs = self.controls()
        for i, c in enumerate(cs):
            if k is None or k == i:
                c.halted = 0
        self.write_controls(cs)

    def run_until(self, t_end: float, chunk: int = 64, max_steps: int = 10 ** 9) -> int:
        """Advance every instance until t >= t_end; returns steps taken (max over instances)."""
        cs = self.controls()
        for c in cs:
            c.t_end = t_end
            c.halted = 0 if c.t < t_end else 1
        self.write_controls(cs)
        start = max(c.step for c in cs)
        while True:
            self.step(chunk)
            cs = self.controls()
            if any(c.status for c in cs):
                self.check()
            steps = max(c.step for c in cs) - start
            if all(c.halted for c in cs) or steps >= max_steps:
                return steps

    # ------------------------------------------------------------------ state
    def state(self, k: int = 0) -> dict[str, torch.Tensor]:
        """Raster views (rows x cols) of the latest state of instance k."""
        cur = self.controls()[k].cur
        ins = self.inst[k]
        out = {"h": ins.raster(ins.h[cur]), "qx": ins.raster(ins.qx[cur]),
               "qy": ins.raster(ins.qy[cur]), "h_max": ins.raster(ins.h_max)}
        if ins.cum is not None:
            out["cum"] = ins.raster(ins.cum)
        z = ins.raster(ins.z).double().cpu().numpy() + ins.z_abs_offset
        out["z"] = torch.as_tensor(z)
        return out

    def compacted(self, k: int = 0) -> dict[str, np.ndarray]:
        """State of instance k in the reference's compacted (row-major valid) order."""
        st = self.state(k)
        v = self.inst[k].valid
        return {name: (t.cpu().numpy() if torch.is_tensor(t) else t)[v].astype(np.float64)
                for name, t in st.items()}

    # ------------------------------------------------------ export / checkpoint
    def time_tag(self, k: int = 0) -> str:
        """The reference's export file tag: str() of the time as a 1-element
        device tensor of the run's dtype (HP/SWE_CUDA.py:836-868 names files
        <field>_<str(t + dt)>.pt; post-processing globs 'h_tensor*.pt')."""
        t = self.controls()[k].t
        return str(torch.tensor([t], dtype=self.dtype, device=self.device))

    def export_fields(self, outpath: str, k: int = 0) -> list[str]:
        """Write h, qx, qy, wl and h_max of instance k as the reference's
        exportField does: compacted (row-major valid-cell order) tensors of the
        run's dtype on the device, one <field>_<tag>.pt file each."""
        ins = self.inst[k]
        st = self.state(k)
        valid = torch.as_tensor(ins.valid, device=self.device)
        z_abs = torch.as_tensor(st["z"], dtype=torch.float64, device=self.device)
        fields = {"h": st["h"], "qx": st["qx"], "qy": st["qy"],
                  "wl": (st["h"].double() + z_abs).to(self.dtype), "h_max": st["h_max"]}
        os.makedirs(outpath, exist_ok=True)
        tag = self.time_tag(k)
        paths = []
        for name, x in fields.items():
            p = os.path.join(outpath, f"{name}_{tag}.pt")
            torch.save(x[valid].contiguous(), p)
            paths.append(p)
        return paths

    def checkpoint(self) -> dict:
        """Device copy of everything a restart needs: each instance's current
        state and h_max, and the control blocks (t, dt, step, export counter,
        rain cursor, volume / rain / outflow totals)."""
        cs = self.controls()
        inst = []
        for k, ins in enumerate(self.inst):
            cur = cs[k].cur
            inst.append({"rows": ins.rows, "cols": ins.cols, "n_valid": ins.n_valid,
                         "h": ins.h[cur].clone(), "qx": ins.qx[cur].clone(),
                         "qy": ins.qy[cur].clone(), "h_max": ins.h_max.clone(),
                         "cum": None if ins.cum is None else ins.cum.clone()})
        return {"dtype": str(self.dtype), "ctrl": self.ctrl.clone(), "instances": inst}

    def restore(self, ckpt: dict) -> None:
        """Resume from checkpoint(): same catchments, same dtype."""
        if ckpt["dtype"] != str(self.dtype) or len(ckpt["instances"]) != len(self.inst):
            raise ValueError("checkpoint does not match this solver (dtype or instances)")
        saved = (_lib.HbCtrl * len(self.inst)).from_buffer_copy(
            bytearray(ckpt["ctrl"].cpu().numpy().tobytes()))
        for k, (ins, rec) in enumerate(zip(self.inst, ckpt["instances"])):
            if (rec["rows"], rec["cols"], rec["n_valid"]) != (ins.rows, ins.cols, ins.n_valid):
                raise ValueError(f"checkpoint instance {k} has another raster")
            cur = saved[k].cur
            ins.h[cur].copy_(rec["h"])
            ins.qx[cur].copy_(rec["qx"])
            ins.qy[cur].copy_(rec["qy"])
            ins.h_max.copy_(rec["h_max"])
            if (ins.cum is None) != (rec.get("cum") is None):
                raise ValueError(f"checkpoint instance {k} differs in infiltration")
            if ins.cum is not None:
                ins.cum.copy_(rec["cum"])
        self.ctrl.copy_(ckpt["ctrl"].to(self.device))
        self.prepare()  # boundary tables and rain rate at t; resets the volume baseline
        cs = self.controls()
        for k, c in enumerate(cs):
            c.volume0 = saved[k].volume0
        self.write_controls(cs)

    def save_checkpoint(self, path: str) -> None:
        ck = self.checkpoint()
        ck["ctrl"] = ck["ctrl"].cpu()
        for rec in ck["instances"]:
            for f in ("h", "qx", "qy", "h_max", "cum"):
                if rec[f] is not None:
                    rec[f] = rec[f].cpu()
        torch.save(ck, path)

    def load_checkpoint(self, path: str) -> None:
        self.restore(torch.load(path, map_location="cpu", weights_only=False))

    def cell_offsets(self, k: int, rows: np.ndarray, cols: np.ndarray) -> torch.Tensor:
        """Flat element offsets of raster cells in the dense state arrays (for gather)."""
        ins = self.inst[k]
        sy, sx = ins.origin
        off = ((np.asarray(rows) + _lib.HB_PAD_Y + sy) * ins.pitch +
               (np.asarray(cols) + _lib.HB_PAD_X + sx))
        return torch.as_tensor(off.astype(np.int64), device=self.device)

    def current(self, k: int = 0) -> tuple[torch.Tensor, torch.Tensor, torch.Tensor]:
        cur = self.controls()[k].cur
        ins = self.inst[k]
        return ins.h[cur], ins.qx[cur], ins.qy[cur]


class HostStepper:
    """Steps a FusedSolver whose state is held in host memory.

    Every step copies h, qx, qy of every instance from pinned host buffers to
    the device, runs one fused step and copies the new h, qx, qy back (the
    host-buffer form of the reference's per-step op calls).  The step always
    reads one fixed device buffer per field (the control block's `cur` is set
    back to it before each step), so the inbound copy of step k+1 runs while
    the outbound copy of step k is still in flight: PCIe carries both
    directions at once.

    layout "compact" (default): the host buffers hold the reference's own
    layout, the valid cells of each instance in row-major order
    (`in_buffers`, `out_buffers`: [h, qx, qy] per instance, views of one
    pinned [3, n_valid] block each, so one copy per instance and direction);
    hb_state_layout moves them between the copied device blocks and the dense
    arrays of the step.  The device blocks are double-buffered (step k uses
    set k % 2), so consecutive copies in one direction follow each other
    without waiting for the step.  Ordering, by CUDA events on three streams:
      * inbound copy k: after the scatter of step k-2 has read its set;
      * scatter k, step k: after inbound copy k (the step's dense input is
        written by scatter k only after step k-1, in stream order);
      * gather k into its outbound set: after outbound copy k-2 has read it;
        outbound copy k: after that gather.
    layout "dense": the host buffers are the padded dense arrays themselves
    (one contiguous copy per field; `raster(buf, k)` is the rows x cols view
    of instance k's cells), the step waiting for the previous outbound copy.
    On the 2048^2 case the dense arrays carry the padding and the tile grid's
    leading no-data columns, about 10 % more bytes than the valid cells.

    Calls are asynchronous: `finish()` makes the caller's stream wait for the
    last outbound copy, after which a synchronize makes `out_buffers` valid.
    """

    def __init__(self, fs: "FusedSolver", layout: str = "compact"):
        if layout not in ("compact", "dense"):
            raise ValueError("layout must be 'compact' or 'dense'")
        self.fs = fs
        self.layout = layout
        dev = fs.device
        cs = fs.controls()
        self.read = cs[0].cur
        if any(c.cur != self.read for c in cs):
            raise ValueError("HostStepper: every instance must read the same buffer index")
        fields = lambda b: [x for ins in fs.inst for x in (ins.h[b], ins.qx[b], ins.qy[b])]
        self._dev_in, self._dev_out = fields(self.read), fields(1 - self.read)
        if layout == "dense":
            self.in_buffers = [torch.empty(x.shape, dtype=x.dtype).pin_memory()
                               for x in self._dev_in]
            self.out_buffers = [torch.empty(x.shape, dtype=x.dtype).pin_memory()
                                for x in self._dev_in]
            for hb, x in zip(self.in_buffers, self._dev_in):
                hb.copy_(x)
        else:
            self._offsets = []
            self._din, self._dout = ([], []), ([], [])  # two device sets each
            self._in_blocks, self._out_blocks = [], []
            for k, ins in enumerate(fs.inst):
                r, c = np.nonzero(ins.valid)
                self._offsets.append(fs.cell_offsets(k, r, c))
                blk = lambda where: (torch.empty((3, r.size), dtype=fs.dtype, device=dev)
                                     if where == "dev" else
                                     torch.empty((3, r.size), dtype=fs.dtype).pin_memory())
                for j in range(2):
                    self._din[j].append(blk("dev"))
                    self._dout[j].append(blk("dev"))
                self._in_blocks.append(blk("host"))
                self._out_blocks.append(blk("host"))
            self.in_buffers = [b[j] for b in self._in_blocks for j in range(3)]
            self.out_buffers = [b[j] for b in self._out_blocks for j in range(3)]
            with torch.cuda.device(dev):
                for k in range(len(fs.inst)):
                    self._layout(k, self._dev_in, self._din[0][k], to_dense=False)
                torch.cuda.current_stream(dev).synchronize()
            for hb, db in zip(self._in_blocks, self._din[0]):
                hb.copy_(db)
        n = len(fs.inst)
        words = fs._ctrl_size // 4
        self._cur = fs.ctrl.view(torch.int32).view(n, words)[:, _lib.HbCtrl.cur.offset // 4]
        self._h2d = torch.cuda.Stream(dev)
        self._d2h = torch.cuda.Stream(dev)
        self._stepped = torch.cuda.Event()
        self._copied_in = torch.cuda.Event()
        self._copied_out = torch.cuda.Event()
        # compact layout: per device set, the scatter that read it, its
        # inbound copy, and the outbound copy that read its gathered result
        self._expanded_set = [torch.cuda.Event(), torch.cuda.Event()]
        self._in_set = [torch.cuda.Event(), torch.cuda.Event()]
        self._out_set = [torch.cuda.Event(), torch.cuda.Event()]
        self._n_steps = 0
        self._any = False

    def _layout(self, k: int, dense: list, block: torch.Tensor, to_dense: bool) -> None:
        fs = self.fs
        h, qx, qy = dense[3 * k:3 * k + 3]
        off = self._offsets[k]
        _lib.check(_lib.lib().hb_state_layout(
            _lib.HB_F32 if fs.dtype == torch.float32 else _lib.HB_F64, off.numel(),
            off.data_ptr(), 1 if to_dense else 0, h.data_ptr(), qx.data_ptr(), qy.data_ptr(),
            block[0].data_ptr(), block[1].data_ptr(), block[2].data_ptr(),
            torch.cuda.current_stream(fs.device).cuda_stream), "hb_state_layout")

    def raster(self, buf: torch.Tensor, k: int = 0) -> torch.Tensor:
        """The rows x cols cells of instance k in one of its host buffers
        (dense layout)."""
        if self.layout != "dense":
            raise ValueError("raster views need layout='dense'; compact buffers are the valid "
                             "cells in row-major order")
        return self.fs.inst[k].raster(buf)

    def step(self) -> None:
        """Enqueue: copy in_buffers to the device, one fused step, copy the
        new state to out_buffers."""
        if self.layout == "dense":
            self._step_dense()
            return
        comp = torch.cuda.current_stream(self.fs.device)
        j = self._n_steps % 2
        din, dout = self._din[j], self._dout[j]
        if self._n_steps >= 2:
            self._h2d.wait_event(self._expanded_set[j])
        with torch.cuda.stream(self._h2d):
            for db, hb in zip(din, self._in_blocks):
                db.copy_(hb, non_blocking=True)
            self._in_set[j].record(self._h2d)
        comp.wait_event(self._in_set[j])
        with torch.cuda.device(self.fs.device):
            for k in range(len(self.fs.inst)):
                self._layout(k, self._dev_in, din[k], to_dense=True)
            self._expanded_set[j].record(comp)
            self._cur.fill_(self.read)
            self.fs.step(1)
            if self._n_steps >= 2:
                comp.wait_event(self._out_set[j])
            for k in range(len(self.fs.inst)):
                self._layout(k, self._dev_out, dout[k], to_dense=False)
        self._stepped.record(comp)
        self._d2h.wait_event(self._stepped)
        with torch.cuda.stream(self._d2h):
            for hb, db in zip(self._out_blocks, dout):
                hb.copy_(db, non_blocking=True)
            self._out_set[j].record(self._d2h)
            self._copied_out.record(self._d2h)
        self._n_steps += 1
        self._any = True

    def _step_dense(self) -> None:
        comp = torch.cuda.current_stream(self.fs.device)
        if self._any:
            self._h2d.wait_event(self._stepped)
        with torch.cuda.stream(self._h2d):
            for x, hb in zip(self._dev_in, self.in_buffers):
                x.copy_(hb, non_blocking=True)
            self._copied_in.record(self._h2d)
        comp.wait_event(self._copied_in)
        if self._any:
            comp.wait_event(self._copied_out)
        self._cur.fill_(self.read)
        self.fs.step(1)
        self._stepped.record(comp)
        self._d2h.wait_event(self._stepped)
        with torch.cuda.stream(self._d2h):
            for hb, x in zip(self.out_buffers, self._dev_out):
                hb.copy_(x, non_blocking=True)
            self._copied_out.record(self._d2h)
        self._any = True

    def finish(self) -> None:
        """Make the caller's current stream wait for the last outbound copy."""
        if self._any:
            torch.cuda.current_stream(self.fs.device).wait_event(self._copied_out)
