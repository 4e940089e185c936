"""GeoTIFF output of raster fields, and GeoTIFF input, with numpy and zlib alone.

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

`read_geotiff` reads one band of a GeoTIFF (the DEM, land-use and rain-mask
rasters the reference opens with rasterio) with its transform, CRS, no-data
value and bounds; `hipims_b200.preprocessing` builds the reference's
pre-processing calls on it.
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


def _raw_geokey_entries(geokeys: dict) -> list:
    """GeoKeyDirectory (34735), GeoDoubleParams (34736) and GeoAsciiParams
    (34737) copied as read from another GeoTIFF: a CRS that is not one EPSG
    code (a user-defined projection, a datum given by parameters) passes
    through unchanged."""
    out = []
    if 34735 in geokeys:
        out.append(_entry(34735, _SHORT, [int(v) for v in geokeys[34735]]))
    if 34736 in geokeys:
        out.append(_entry(34736, _DOUBLE, [float(v) for v in geokeys[34736]]))
    if 34737 in geokeys:
        txt = geokeys[34737]
        if isinstance(txt, bytes):
            txt = txt.decode("ascii", "replace")
        out.append(_entry(34737, _ASCII, str(txt).rstrip("\0")))
    return out


def _geo_entries(transform, epsg: int | None, geographic: bool | None,
                 geokeys: dict | None = None) -> list:
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
    if geokeys:
        return out + _raw_geokey_entries(geokeys)
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
                  geographic: bool | None = None, geokeys: dict | None = None) -> str:
    """Write a 2-D array as a single-band float32 GeoTIFF (little-endian,
    uncompressed, one strip).  epsg: the CRS as an EPSG code (a projected CRS
    unless the code is a known geographic one or `geographic` says so);
    geokeys: the GeoKey tags of another GeoTIFF ({34735: ..., 34736: ...,
    34737: ...}, as read_geotiff returns them in meta["geokeys"]), written
    verbatim instead."""
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
    entries += _geo_entries(transform, epsg, geographic, geokeys)
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
                       geokeys: dict | None = None,
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
        out.append(write_geotiff(reference_tif_name(p), raster, transform, epsg, nodata,
                                 geokeys=geokeys))
    return out


# ---------------------------------------------------------------------------
# Reading (the reference opens its DEM, land-use and rain-mask rasters with
# rasterio: `src.read(1, masked=True)` and `src.meta`, HP/preProcessing.py:
# 140-143, 228-230, 354-357, 382-385)
# ---------------------------------------------------------------------------

# TIFF field types: struct code and size in bytes
_FIELD = {1: ("B", 1), 2: ("s", 1), 3: ("H", 2), 4: ("I", 4), 5: ("I", 8), 6: ("b", 1),
          7: ("B", 1), 8: ("h", 2), 9: ("i", 4), 10: ("i", 8), 11: ("f", 4), 12: ("d", 8),
          16: ("Q", 8), 17: ("q", 8), 18: ("Q", 8)}


def _ifd(buf: bytes, off: int, bo: str, big: bool) -> dict:
    """Tags of the image file directory at `off`: tag -> list of values
    (a str for ASCII, bytes for UNDEFINED)."""
    n = struct.unpack_from(bo + ("Q" if big else "H"), buf, off)[0]
    off += 8 if big else 2
    size, inline = (20, 8) if big else (12, 4)
    tags = {}
    for k in range(n):
        e = off + k * size
        tag, typ, cnt = struct.unpack_from(bo + ("HHQ" if big else "HHI"), buf, e)
        if typ not in _FIELD:
            continue
        code, width = _FIELD[typ]
        nbytes = width * cnt
        at = e + (12 if big else 8)
        if nbytes > inline:
            at = struct.unpack_from(bo + ("Q" if big else "I"), buf, at)[0]
        raw = buf[at:at + nbytes]
        if typ == 2:
            tags[tag] = raw.split(b"\0")[0].decode("latin-1")
        elif typ == 7:
            tags[tag] = bytes(raw)
        elif typ in (5, 10):  # rationals: numerator / denominator pairs
            v = struct.unpack(bo + code * (2 * cnt), raw)
            tags[tag] = [v[2 * i] / v[2 * i + 1] if v[2 * i + 1] else float("nan")
                         for i in range(cnt)]
        else:
            tags[tag] = list(struct.unpack(bo + code * cnt, raw))
    return tags


def _lzw_decode(data: bytes) -> bytes:
    """TIFF LZW (codes written most significant bit first, 9 to 12 bits, 256
    clears the table, 257 ends the strip, the code width grows one code early)."""
    out = bytearray()
    table = [bytes((i,)) for i in range(256)] + [b"", b""]
    bits, acc, nacc, prev = 9, 0, 0, None
    it = iter(data)
    while True:
        while nacc < bits:
            byte = next(it, None)
            if byte is None:
                return bytes(out)
            acc = (acc << 8) | byte
            nacc += 8
        nacc -= bits
        code = (acc >> nacc) & ((1 << bits) - 1)
        acc &= (1 << nacc) - 1
        if code == 256:
            del table[258:]
            bits, prev = 9, None
            continue
        if code == 257:
            return bytes(out)
        if prev is None:
            entry = table[code]
        else:
            entry = table[code] if code < len(table) else prev + prev[:1]
            if len(table) < 4096:
                table.append(prev + entry[:1])
        out += entry
        prev = entry
        if len(table) >= (1 << bits) - 1 and bits < 12:
            bits += 1


def _packbits_decode(data: bytes) -> bytes:
    out = bytearray()
    i, n = 0, len(data)
    while i < n:
        c = data[i]
        i += 1
        if c < 128:  # c + 1 literal bytes
            out += data[i:i + c + 1]
            i += c + 1
        elif c > 128:  # the next byte 257 - c times
            out += bytes((data[i],)) * (257 - c)
            i += 1
    return bytes(out)


def _decompress(raw: bytes, compression: int) -> bytes:
    import zlib

    if compression == 1:
        return raw
    if compression in (8, 32946):
        return zlib.decompress(raw)
    if compression == 5:
        return _lzw_decode(raw)
    if compression == 32773:
        return _packbits_decode(raw)
    raise ValueError(f"TIFF compression {compression} is not supported "
                     "(none, LZW, deflate and PackBits are)")


def _sample_dtype(bits: int, fmt: int, bo: str) -> np.dtype:
    kind = {1: "u", 2: "i", 3: "f"}.get(fmt)
    if kind is None or bits not in (8, 16, 32, 64) or (kind == "f" and bits < 32):
        raise ValueError(f"TIFF samples of {bits} bits, format {fmt}, are not supported")
    return np.dtype(("<" if bo == "<" else ">") + kind + str(bits // 8))


def _unpredict(block: np.ndarray, predictor: int, dtype: np.dtype, spp: int) -> np.ndarray:
    """Undo the predictor on a chunk of rows x n samples (n = columns x spp).
    2: horizontal differences, sample by sample; 3: the floating-point
    predictor (each row's bytes grouped by significance, most significant
    group first, then byte-wise differences with a stride of spp)."""
    rows, n = block.shape
    if predictor == 2:
        v = block.reshape(rows, n // spp, spp)
        if dtype.kind == "f":
            return np.cumsum(v, axis=1, dtype=dtype).reshape(rows, n)
        wide = np.uint64 if dtype.kind == "u" else np.int64
        return np.cumsum(v.astype(wide), axis=1).astype(dtype).reshape(rows, n)
    if predictor == 3:
        w = dtype.itemsize
        b = np.ascontiguousarray(block).view(np.uint8).reshape(rows, n * w)
        b = np.cumsum(b.reshape(rows, -1, spp), axis=1, dtype=np.uint8).reshape(rows, n * w)
        be = np.ascontiguousarray(b.reshape(rows, w, n).transpose(0, 2, 1))
        return be.view(np.dtype(">" + dtype.kind + str(w))).reshape(rows, n)
    return block


def read_geotiff(path: str, band: int = 1, masked: bool = False):
    """One band of a GeoTIFF and its metadata, without rasterio or GDAL.

    Classic or BigTIFF, either byte order; strips or tiles; no compression,
    LZW, deflate or PackBits; predictors 2 and 3; 8-64-bit integer or 32/64-bit
    float samples, interleaved or planar.  Returns (array, meta): meta holds
    the keys of rasterio's `src.meta` (driver, dtype, nodata, width, height,
    count, crs as 'EPSG:<code>' or None, transform as the affine tuple
    (a, b, c, d, e, f)) and `bounds` (left, bottom, right, top).  masked=True
    returns a numpy masked array whose mask marks the no-data cells, as
    rasterio's `read(band, masked=True)`."""
    with open(path, "rb") as fh:
        buf = fh.read()
    bo = {b"II": "<", b"MM": ">"}.get(buf[:2])
    if bo is None:
        raise ValueError(f"{path}: not a TIFF file")
    magic = struct.unpack_from(bo + "H", buf, 2)[0]
    if magic == 42:
        big, first = False, struct.unpack_from(bo + "I", buf, 4)[0]
    elif magic == 43:
        big, first = True, struct.unpack_from(bo + "Q", buf, 8)[0]
    else:
        raise ValueError(f"{path}: not a TIFF file")
    t = _ifd(buf, first, bo, big)
    width, height = int(t[256][0]), int(t[257][0])
    spp = int(t.get(277, [1])[0])
    bits = int(t.get(258, [1])[0])
    fmt = int(t.get(339, [1])[0])
    comp = int(t.get(259, [1])[0])
    predictor = int(t.get(317, [1])[0])
    planar = int(t.get(284, [1])[0])
    if not 1 <= band <= spp:
        raise ValueError(f"{path}: band {band} of {spp}")
    dtype = _sample_dtype(bits, fmt, bo)
    chunky = spp if planar == 1 else 1
    if 322 in t:  # tiles
        cw, ch = int(t[322][0]), int(t[323][0])
        offsets, counts = t[324], t[325]
    else:
        cw, ch = width, int(t.get(278, [height])[0])
        ch = min(ch, height)
        offsets, counts = t[273], t[279]
    across, down = -(-width // cw), -(-height // ch)
    per_plane = across * down
    out = np.empty((height, width), dtype=dtype.newbyteorder("="))
    first_chunk = (band - 1) * per_plane if planar == 2 else 0
    for k in range(per_plane):
        raw = buf[offsets[first_chunk + k]:offsets[first_chunk + k] + counts[first_chunk + k]]
        data = _decompress(raw, comp)
        rows_here = ch if 322 in t else min(ch, height - (k // across) * ch)
        need = rows_here * cw * chunky * dtype.itemsize
        block = np.frombuffer(data[:need], dtype=dtype).reshape(rows_here, cw * chunky)
        block = _unpredict(block, predictor, dtype, chunky).astype(dtype.newbyteorder("="))
        if chunky > 1:
            block = block.reshape(rows_here, cw, chunky)[:, :, band - 1]
        r0, c0 = (k // across) * ch, (k % across) * cw
        r1, c1 = min(r0 + rows_here, height), min(c0 + cw, width)
        out[r0:r1, c0:c1] = block[:r1 - r0, :c1 - c0]
    meta = _geo_meta(t, width, height, spp, out.dtype)
    if masked:
        nd = meta["nodata"]
        if nd is None:
            mask = np.zeros(out.shape, dtype=bool)
        elif np.isnan(nd):
            mask = np.isnan(out)
        else:
            mask = out == np.asarray(nd).astype(out.dtype)
        return np.ma.MaskedArray(out, mask=mask), meta
    return out, meta


def _geo_meta(t: dict, width: int, height: int, count: int, dtype) -> dict:
    transform = None
    if 34264 in t:
        m = t[34264]
        transform = (m[0], m[1], m[3], m[4], m[5], m[7])
    elif 33550 in t and 33922 in t:
        sx, sy = t[33550][0], t[33550][1]
        i, j, x, y = t[33922][0], t[33922][1], t[33922][3], t[33922][4]
        transform = (sx, 0.0, x - i * sx, 0.0, -sy, y + j * sy)
    keys = {}
    if 34735 in t:
        d = t[34735]
        for q in range(d[3]):
            kid, loc, _, val = d[4 + 4 * q:8 + 4 * q]
            if loc == 0:
                keys[kid] = val
    if transform is not None and keys.get(1025) == 2:
        # PixelIsPoint: the tie point is a pixel centre; GDAL's default moves
        # the origin half a pixel to the corner
        a, b, c, d_, e, f = transform
        transform = (a, b, c - 0.5 * a - 0.5 * b, d_, e, f - 0.5 * d_ - 0.5 * e)
    # 32767 marks a user-defined CRS (its parameters are in other keys), not an EPSG code
    epsg = next((keys[k] for k in (3072, 2048) if keys.get(k) not in (None, 0, 32767)), None)
    nodata = None
    if 42113 in t:
        try:
            nodata = float(t[42113].strip())
        except ValueError:
            nodata = None
    bounds = None
    if transform is not None:
        a, b, c, d_, e, f = transform
        xs = [c, c + a * width, c + b * height, c + a * width + b * height]
        ys = [f, f + d_ * width, f + e * height, f + d_ * width + e * height]
        bounds = (min(xs), min(ys), max(xs), max(ys))
    geokeys = {k: t[k] for k in (34735, 34736, 34737) if k in t}
    return dict(driver="GTiff", dtype=str(np.dtype(dtype)), nodata=nodata, width=width,
                height=height, count=count, crs=f"EPSG:{epsg}" if epsg else None,
                transform=transform, bounds=bounds, geokeys=geokeys)
