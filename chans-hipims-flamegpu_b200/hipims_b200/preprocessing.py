"""Raster inputs of a run: DEM, boundary coding, gauges, land use and rain
mask, read from GeoTIFF files without rasterio.

The functions keep the names, arguments and return values of the reference's
pre-processing (HP/preProcessing.py:140-177, 221-348, 354-390), so a driver
written against it runs unchanged.  The files are read by
`hipims_b200.geotiff.read_geotiff`; `demMeta['transform']` is the affine
tuple (a, b, c, d, e, f), which indexes like rasterio's Affine.

Differences from the reference, none on well-formed inputs:
  * a box of type FALL (9) is coded like the others (the reference's id
    counter has no slot for it and raises IndexError);
  * an unknown boundary-type name raises ValueError (the reference prints the
    valid names and goes on with an unset type);
  * one type code or name for every box is accepted as well as one per box;
  * boundBox is not clipped in place (the reference writes the clipped
    corners back into the caller's array).
"""
from __future__ import annotations

from typing import Sequence

import numpy as np
import torch

from .geotiff import read_geotiff

BC_TYPES = {"RIGID": 3, "WALL_SLIP": 4, "OPEN": 5, "H_GIVEN": 6, "Q_GIVEN": 7, "WL_GIVEN": 8,
            "FALL": 9}
# neighbour shifts of the boundary ring (torch.roll shift, dim), as
# HP/preProcessing.py:158, 239
_RING_ROLLS = ((-1, 1), (1, 0), (1, 1), (-1, 0))


def rowcol(transform: Sequence[float], xs, ys) -> tuple[np.ndarray, np.ndarray]:
    """Raster row and column of map positions (rasterio.transform.rowcol with
    its default floor): the pixel whose area holds each point."""
    a, b, c, d, e, f = (float(v) for v in transform[:6])
    x = np.asarray(xs, dtype=np.float64) - c
    y = np.asarray(ys, dtype=np.float64) - f
    det = a * e - b * d
    col = (e * x - b * y) / det
    row = (-d * x + a * y) / det
    return np.floor(row).astype(np.int64), np.floor(col).astype(np.int64)


def _ring(nodata: np.ndarray) -> np.ndarray:
    """Valid cells with a no-data 4-neighbour (the raster wraps, as torch.roll)."""
    nd = nodata.astype(np.int32)
    ring = np.zeros_like(nd)
    for shift, dim in _RING_ROLLS:
        ring += np.roll(nd, shift, axis=dim)
    ring[nodata] = 0
    return ring.astype(bool)


def importDEMData(DEM_path: str, device):
    """(dem, mask, mask_boundary, demMeta) as HP/preProcessing.py:140-177:
    dem with no-data filled by -9999, mask True on valid cells, mask_boundary
    True on valid cells with a no-data neighbour."""
    demMasked, demMeta = read_geotiff(DEM_path, masked=True)
    dem = np.ma.filled(demMasked, fill_value=-9999.0)
    nodata = np.ma.getmaskarray(demMasked)
    boundary = _ring(nodata)
    return (torch.from_numpy(dem).to(device=device), torch.from_numpy(~nodata).to(device=device),
            torch.from_numpy(boundary).to(device=device), demMeta)


def importDEMData_And_BC(DEM_path: str, device, gauges_position=np.array([]),
                         boundBox=np.array([]), default_BC: int = 50, bc_type=5):
    """(dem, mask, demMeta, gauge_index_1D) as HP/preProcessing.py:221-348.

    mask (int32): 0 on no-data, 1 inside, `default_BC` on the boundary ring;
    ring cells inside boundBox[i] = (left, bottom, right, top), in map units
    and clipped to the raster's bounds, get int(str(type) + str(id)) with
    type bc_type[i] (a code 3-9 or a name of BC_TYPES) and id counting the
    boxes of that type from 0 (from 1 when the default code has that type).
    gauge_index_1D (int64): the compacted index (row-major order of the
    valid cells) of each gauge position (x, y), in the order given."""
    demMasked, demMeta = read_geotiff(DEM_path, masked=True)
    dem = np.ma.filled(demMasked, fill_value=-9999.0)
    nodata = np.ma.getmaskarray(demMasked)
    boundary = _ring(nodata)
    mask = (~nodata).astype(np.int32)

    gauge_index_1D = torch.tensor([])
    gauges_position = np.asarray(gauges_position)
    if gauges_position.size > 0:
        rows, cols = rowcol(demMeta["transform"], gauges_position[:, 0], gauges_position[:, 1])
        mask_gauge = mask.copy()
        mask_gauge[rows, cols] = 100
        marked = mask_gauge[mask_gauge > 0] >= 99
        idx = torch.from_numpy(np.flatnonzero(marked)).to(torch.int64)
        # the reference's reordering into the order of the given positions
        order = (rows * dem.shape[1] + cols).argsort()
        ranks = order.argsort()
        gauge_index_1D = idx[torch.from_numpy(ranks)]

    mask[boundary] = default_BC
    count = {t: -1 for t in BC_TYPES.values()}
    count[int(str(default_BC)[0])] += 1
    boundBox = np.asarray(boundBox, dtype=np.float64)
    if boundBox.size > 0:
        left, bottom, right, top = demMeta["bounds"]
        for i in range(len(boundBox)):
            t = bc_type[i] if isinstance(bc_type, (list, tuple, np.ndarray)) else bc_type
            if isinstance(t, str):
                if t not in BC_TYPES:
                    raise ValueError(f"boundary type {t!r}: the names are {', '.join(BC_TYPES)}")
                t = BC_TYPES[t]
            t = int(t)
            box = boundBox[i].copy()
            box[0], box[1] = max(left, box[0]), max(bottom, box[1])
            box[2], box[3] = min(right, box[2]), min(top, box[3])
            rows_min, cols_min = rowcol(demMeta["transform"], box[0], box[1])
            rows_max, cols_max = rowcol(demMeta["transform"], box[2], box[3])
            in_box = np.zeros(mask.shape, dtype=bool)
            # rows run from the top down, so the top edge gives the first row
            in_box[int(rows_max):int(rows_min), int(cols_min):int(cols_max)] = True
            count[t] += 1
            mask[boundary & in_box] = int(f"{t}{count[t]}")

    return (torch.from_numpy(dem).to(device=device), torch.from_numpy(mask).to(device=device),
            demMeta, gauge_index_1D)


def importLanduseData(LandUse_path: str, device, level: int = 0):
    """(landuse, landuse_index) as HP/preProcessing.py:354-379: no-data filled
    with 1; level 1 maps a code c to int(c / 10) - 1 (no-data: 11 -> 0);
    otherwise the k-th smallest code (k >= 1) becomes k - 1, in place and in
    order, the smallest code keeping its value."""
    masked, _ = read_geotiff(LandUse_path, masked=True)
    if level == 1:
        landuse = np.ma.filled(masked, fill_value=11)
        landuse = (landuse / 10).astype(int) - 1
        classes = len(np.unique(landuse)) - 1
        out = torch.from_numpy(landuse).to(device=device)
    else:
        landuse = np.ma.filled(masked, fill_value=1)
        classes = len(np.unique(landuse)) - 1
        indexes = np.unique(landuse)
        out = torch.from_numpy(landuse).to(device=device)
        for i in range(1, len(indexes)):
            out[out == indexes[i]] = i - 1
    return out, np.arange(classes)


def importRainStationMask(rainmask_path: str, device):
    """The rain-station index of every cell (int16; no-data -> station 0), as
    HP/preProcessing.py:382-390."""
    masked, _ = read_geotiff(rainmask_path, masked=True)
    rainmask = np.ma.filled(masked, fill_value=0).astype(np.int16)
    return torch.from_numpy(rainmask).to(device=device)
