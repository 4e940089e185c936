"""Raster topology: compaction, neighbour table and boundary coding.

* compact_index restates HP/SWE_CUDA.py:173-222 (``init__fluidField_tensor``):
  valid cells are ``mask > 0`` in row-major order; ``index`` is [5, N] int32
  flattened, row 0 the cell's type code, rows 1-4 the compacted ids of the E,
  N (row - 1), W and S (row + 1) neighbours or -1.  Neighbours come from
  ``torch.roll`` and therefore wrap around the raster edge, as in the
  reference, which is why rasters carry a no-data outer ring.
* boundary_codes restates the coding of HP/preProcessing.py:221-348: valid
  cells with a no-data 4-neighbour form the boundary ring and get
  ``default_bc``; interior cells get 1; boxes get ``int(str(type) + str(k))``
  with k counting boxes of the same type (starting after the default).
  Types: RIGID 3, WALL_SLIP 4, OPEN 5, H_GIVEN 6, Q_GIVEN 7, WL_GIVEN 8, FALL 9.
* decode_bc restates the kernels' decode (HC/flucCal_2ndOrder_jh_improved_
  Kernel.cu:430-438): leading decimal digit = type, remaining digits = id.
"""
from __future__ import annotations

import numpy as np
import torch

BC_TYPES = {"RIGID": 3, "WALL_SLIP": 4, "OPEN": 5, "H_GIVEN": 6, "Q_GIVEN": 7,
            "WL_GIVEN": 8, "FALL": 9}

# torch.roll arguments of HP/SWE_CUDA.py:183 giving E, N, W, S neighbours
_ROLLS = ((-1, 1), (1, 0), (1, 1), (-1, 0))


def decode_bc(code: int) -> tuple[int, int]:
    code = int(code)
    bt, p = code, 1
    while bt >= 10:
        bt //= 10
        p *= 10
    return bt, code - bt * p


def compact_index(mask: torch.Tensor) -> torch.Tensor:
    """Flattened [5 * N] int32 neighbour table of a raster of type codes."""
    valid = mask > 0
    n = int(valid.sum())
    ids = torch.full(mask.shape, -1, dtype=torch.int32, device=mask.device)
    ids[valid] = torch.arange(n, dtype=torch.int32, device=mask.device)
    index = torch.empty((5, n), dtype=torch.int32, device=mask.device)
    index[0] = mask[valid].to(torch.int32)
    for d, (shift, dim) in enumerate(_ROLLS):
        index[d + 1] = ids.roll(shift, dim)[valid]
    return index.flatten()


def compact(mask: torch.Tensor, field: torch.Tensor, dtype=None) -> torch.Tensor:
    """field[mask > 0] in row-major order (the reference's state layout)."""
    out = field[mask > 0]
    return out.to(dtype) if dtype is not None else out.clone()


def boundary_codes(nodata: np.ndarray, default_bc: int = 50,
                   boxes: list[tuple[int, int, int, int, int]] | None = None) -> np.ndarray:
    """int32 raster of type codes (<= 0 for no-data, here -9999).

    boxes: (row0, row1, col0, col1, type) half-open raster index ranges; only
    boundary-ring cells inside a box are recoded.
    """
    nodata = np.asarray(nodata, dtype=bool)
    nd = nodata.astype(np.int32)
    ring = np.zeros_like(nd)
    for shift, dim in _ROLLS:
        ring += np.roll(nd, shift, axis=dim)
    ring[nodata] = 0
    ring = ring.astype(bool)
    code = np.where(nodata, -9999, 1).astype(np.int32)
    code[ring] = default_bc
    count = {t: -1 for t in BC_TYPES.values()}
    count[int(str(default_bc)[0])] += 1
    for (r0, r1, c0, c1, btype) in boxes or []:
        box = np.zeros_like(nodata)
        box[r0:r1, c0:c1] = True
        count[btype] += 1
        code[ring & box] = int(f"{btype}{count[btype]}")
    return code


def compacted_positions(mask: torch.Tensor) -> torch.Tensor:
    """(row, col) of each compacted cell, [N, 2] int64, row-major order."""
    return torch.nonzero(mask > 0)
