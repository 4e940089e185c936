"""GeoTIFF output of raster fields, written with numpy alone.

The reference writes its results with rasterio (HP/postProcessing.py:26-196,
`exportRaster_tiff`): every exported field file (`<field>_<str(t)>.pt`, a
compacted vector of the valid cells) is scattered into the DEM's raster,
no-data cells are filled with -9999, and the raster is written as a float32
GeoTIFF with the DEM's georeferencing under the name `<prefix>_<time>tif`.
rasterio and GDAL are not needed here: `write_geotiff` writes a baseline
TIFF (one float32 band, uncompressed, one strip) carrying the GeoTIFF tags
that GDAL and rasterio read back as the transform, the CRS (an EPSG code)
and the no-data value.

    write_geotiff("h_max.tif", h_max, transform=(2.0, 0.0, 500000.0,
                  0.0, -2.0, 4200000.0), epsg=27700)
    export_raster_tiff("out", mask, transform=..., epsg=27700)

`transform` is rasterio's affine order (a, b, c, d, e, f): the map position
of the upper-left corner of pixel (row, col) is x = a col + b row + c,
y = d col + e row + f (a 9-element sequence, as tuple(Affine) gives, is
accepted too).
"""
from __future__ import annotations

import glob
import os
import struct
from typing import Sequence

import numpy as np

_SHORT, _LONG, _DOUBLE, _ASCII = 3, 4, 12, 2
GEOGRAPHIC_EPSG = frozenset({4326, 4269, 4258, 4283, 4612, 4167, 4152, 4619})


def _entry(tag: int, typ: int, values) -> tuple[int, int, int, bytes]:
    if typ == _ASCII:
        data = values.encode("ascii") + b"\0"
        return tag, typ, len(data), data
    fmt = {_SHORT: "H", _LONG: "I", _DOUBLE: "d"}[typ]
    values = list(values)
    return tag, typ, len(values), struct.pack("<" + fmt * len(values), *values)


def _geo_entries(transform, epsg: int | None, geographic: bool | None) -> list:
    out = []
    if transform is not None:
        t = [float(v) for v in transform]
        if len(t) == 9:
            t = t[:6]
        if len(t) != 6:
            raise ValueError("transform: 6 (or 9) affine coefficients a, b, c, d, e, f")
        a, b, c, d, e, f = t
        if b == 0.0 and d == 0.0:
            out.append(_entry(33550, _DOUBLE, (a, -e, 0.0)))             # ModelPixelScale
            out.append(_entry(33922, _DOUBLE, (0.0, 0.0, 0.0, c, f, 0.0)))  # ModelTiepoint
        else:
            out.append(_entry(34264, _DOUBLE, (a, b, 0.0, c, d, e, 0.0, f,  # ModelTransformation
                                               0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 1.0)))
    keys = []
    if epsg is not None:
        geo = (int(epsg) in GEOGRAPHIC_EPSG) if geographic is None else bool(geographic)
        keys.append((1024, 2 if geo else 1))               # GTModelType
        keys.append((1025, 1))                             # GTRasterType: PixelIsArea
        keys.append((2048 if geo else 3072, int(epsg)))    # Geographic / ProjectedCSType
    elif transform is not None:
        keys.append((1025, 1))
    if keys:
        d = [1, 1, 0, len(keys)]
        for kid, val in keys:
            d += [kid, 0, 1, val]
        out.append(_entry(34735, _SHORT, d))               # GeoKeyDirectory
    return out


def write_geotiff(path: str, data, transform: Sequence[float] | None = None,
                  epsg: int | None = None, nodata: float | None = -9999.0,
                  geographic: bool | None = None) -> str:
    """Write a 2-D array as a single-band float32 GeoTIFF (little-endian,
    uncompressed, one strip).  epsg: the CRS as an EPSG code (a projected CRS
    unless the code is a known geographic one or `geographic` says so)."""
    arr = np.ascontiguousarray(np.asarray(data), dtype="<f4")
    if arr.ndim != 2:
        raise ValueError("write_geotiff: a 2-D raster")
    rows, cols = arr.shape
    nbytes = arr.nbytes
    if nbytes + 4096 >= 2 ** 32:
        raise ValueError("write_geotiff: rasters of 4 GiB or more need BigTIFF")
    data_off = 8
    entries = [
        _entry(256, _LONG, [cols]), _entry(257, _LONG, [rows]), _entry(258, _SHORT, [32]),
        _entry(259, _SHORT, [1]), _entry(262, _SHORT, [1]), _entry(273, _LONG, [data_off]),
        _entry(277, _SHORT, [1]), _entry(278, _LONG, [rows]), _entry(279, _LONG, [nbytes]),
        _entry(284, _SHORT, [1]), _entry(339, _SHORT, [3]),
    ]
    entries += _geo_entries(transform, epsg, geographic)
    if nodata is not None:
        entries.append(_entry(42113, _ASCII, "%.17g" % float(nodata)))  # GDAL_NODATA
    entries.sort(key=lambda x: x[0])
    ifd_off = data_off + nbytes + (nbytes & 1)
    ifd_size = 2 + 12 * len(entries) + 4
    ifd, extra = bytearray(struct.pack("<H", len(entries))), bytearray()
    for tag, typ, count, payload in entries:
        if len(payload) <= 4:
            ifd += struct.pack("<HHI", tag, typ, count) + payload.ljust(4, b"\0")
        else:
            ifd += struct.pack("<HHII", tag, typ, count, ifd_off + ifd_size + len(extra))
            extra += payload
            if len(extra) & 1:
                extra += b"\0"
    ifd += struct.pack("<I", 0)
    with open(path, "wb") as f:
        f.write(b"II" + struct.pack("<HI", 42, ifd_off))
        f.write(arr.tobytes())
        if nbytes & 1:
            f.write(b"\0")
        f.write(bytes(ifd))
        f.write(bytes(extra))
    return path


def reference_tif_name(pt_path: str) -> str:
    """The reference's output name for an exported field file
    (HP/postProcessing.py:190-193): the path up to its last '_', then '_',
    then the text between '[' and ']' of the time tag, then 'tif'.  For a time
    printed with a trailing '.' (`tensor([3600.], ...)`) that gives
    `h_3600.tif`; a fractional time gives `h_3600.5000tif`, as the reference
    does."""
    top = pt_path[:pt_path.rfind("_")]
    t = pt_path[pt_path.find("[") + 1:pt_path.find("]")]
    return top + "_" + t + "tif"


def export_raster_tiff(outpath: str, mask, transform: Sequence[float] | None = None,
                       epsg: int | None = None, nodata: float = -9999.0,
                       pattern: str = "*.pt") -> list[str]:
    """GeoTIFFs of every exported field file in `outpath`
    (`FusedSolver.export_fields`, `Godunov.exportField`): the compacted vector
    goes to the valid cells of `mask` (> 0, row-major), every other cell gets
    `nodata`; names as `reference_tif_name`."""
    import torch

    valid = np.asarray(mask) > 0
    out = []
    for p in sorted(glob.glob(os.path.join(outpath, pattern))):
        vec = torch.load(p, map_location="cpu", weights_only=False)
        vec = np.asarray(vec.detach().cpu().numpy() if hasattr(vec, "detach") else vec)
        if vec.shape != (int(valid.sum()),):
            raise ValueError(f"{p}: {vec.shape[0]} values for {int(valid.sum())} valid cells")
        raster = np.full(valid.shape, nodata, dtype=np.float32)
        raster[valid] = vec.astype(np.float32)
        out.append(write_geotiff(reference_tif_name(p), raster, transform, epsg, nodata))
    return out
