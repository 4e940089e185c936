"""GeoTIFF input without rasterio (hipims_b200.geotiff.read_geotiff): files
written by Pillow's libtiff (every compression and predictor it offers), by
this package's writer (georeferencing and no-data), and by a small writer
here for the layouts Pillow does not make (tiles with ragged edge tiles,
several strips, big-endian, BigTIFF, interleaved and planar bands)."""
import struct
import zlib

import numpy as np
import pytest
from PIL import Image

from hipims_b200.geotiff import read_geotiff, write_geotiff


def _pillow(path, a, compression=None, predictor=None):
    info = {317: predictor} if predictor else {}
    Image.fromarray(a).save(path, format="TIFF", compression=compression, tiffinfo=info)


@pytest.mark.parametrize("compression,predictor", [
    (None, None), ("tiff_lzw", None), ("tiff_adobe_deflate", None), ("packbits", None),
    ("tiff_adobe_deflate", 3), ("tiff_lzw", 3)])
def test_float32_from_libtiff(tmp_path, compression, predictor):
    a = (np.random.default_rng(1).normal(size=(53, 71)) * 100).astype(np.float32)
    p = str(tmp_path / "f.tif")
    _pillow(p, a, compression, predictor)
    got, meta = read_geotiff(p)
    assert got.dtype == np.float32 and meta["width"] == 71 and meta["height"] == 53
    np.testing.assert_array_equal(got, a)


@pytest.mark.parametrize("dtype", [np.uint8, np.uint16, np.int32])
@pytest.mark.parametrize("compression", ["tiff_lzw", "tiff_adobe_deflate"])
def test_integers_with_horizontal_predictor(tmp_path, dtype, compression):
    a = np.random.default_rng(2).integers(0, 250, size=(40, 33)).astype(dtype)
    p = str(tmp_path / "i.tif")
    _pillow(p, a, compression, 2)
    got, _ = read_geotiff(p)
    assert got.dtype == dtype
    np.testing.assert_array_equal(got, a)


def test_lzw_long_strip_resets_its_table(tmp_path):
    """Enough distinct data that the LZW table fills and is cleared."""
    a = np.random.default_rng(3).integers(0, 256, size=(300, 300)).astype(np.uint8)
    p = str(tmp_path / "l.tif")
    _pillow(p, a, "tiff_lzw")
    np.testing.assert_array_equal(read_geotiff(p)[0], a)


def test_own_writer_round_trip_with_georeferencing(tmp_path):
    a = np.random.default_rng(4).uniform(0, 50, size=(30, 20)).astype(np.float32)
    a[0, :] = -9999.0
    p = write_geotiff(str(tmp_path / "g.tif"), a, transform=(2.0, 0.0, 500000.0, 0.0, -2.0,
                                                              4200000.0), epsg=27700)
    got, meta = read_geotiff(p, masked=True)
    np.testing.assert_array_equal(got.data, a)
    assert got.mask[0].all() and not got.mask[1:].any()
    assert meta["transform"] == (2.0, 0.0, 500000.0, 0.0, -2.0, 4200000.0)
    assert meta["crs"] == "EPSG:27700" and meta["nodata"] == -9999.0
    assert meta["bounds"] == (500000.0, 4200000.0 - 60.0, 500040.0, 4200000.0)
    # a rotated/sheared transform goes through ModelTransformation
    t = (1.5, 0.25, 100.0, -0.25, -1.5, 900.0)
    p2 = write_geotiff(str(tmp_path / "r.tif"), a, transform=t, epsg=4326)
    _, m2 = read_geotiff(p2)
    assert m2["transform"] == t and m2["crs"] == "EPSG:4326"


def _write_tiff(path, a, bo="<", big=False, tile=None, rows_per_strip=None, planar=1,
                deflate=False):
    """A minimal TIFF writer: a (H, W) or (H, W, S) array, strips or tiles,
    optional deflate, either byte order, classic or BigTIFF."""
    a = np.asarray(a)
    if a.ndim == 2:
        a = a[:, :, None]
    H, W, S = a.shape
    dt = a.dtype.newbyteorder(bo)
    fmt = {"u": 1, "i": 2, "f": 3}[a.dtype.kind]
    chunks = []
    planes = [a] if planar == 1 else [a[:, :, s:s + 1] for s in range(S)]
    for pl in planes:
        if tile:
            tw, th = tile
            for r0 in range(0, H, th):
                for c0 in range(0, W, tw):
                    t = np.zeros((th, tw, pl.shape[2]), dtype=a.dtype)
                    blk = pl[r0:r0 + th, c0:c0 + tw]
                    t[:blk.shape[0], :blk.shape[1]] = blk
                    chunks.append(t.astype(dt).tobytes())
        else:
            rps = rows_per_strip or H
            for r0 in range(0, H, rps):
                chunks.append(pl[r0:r0 + rps].astype(dt).tobytes())
    if deflate:
        chunks = [zlib.compress(c) for c in chunks]
    head = 16 if big else 8
    offsets, pos = [], head
    for c in chunks:
        offsets.append(pos)
        pos += len(c)
    LONGT = 16 if big else 4
    entries = [(256, 4, [W]), (257, 4, [H]), (258, 3, [a.dtype.itemsize * 8] * S),
               (259, 3, [8 if deflate else 1]), (262, 3, [1]), (277, 3, [S]),
               (284, 3, [planar]), (339, 3, [fmt] * S)]
    if tile:
        entries += [(322, 4, [tile[0]]), (323, 4, [tile[1]]), (324, LONGT, offsets),
                    (325, LONGT, [len(c) for c in chunks])]
    else:
        entries += [(273, LONGT, offsets), (278, 4, [rows_per_strip or H]),
                    (279, LONGT, [len(c) for c in chunks])]
    entries.sort()
    code = {3: "H", 4: "I", 16: "Q"}
    esize, inline = (20, 8) if big else (12, 4)
    ifd_at = pos
    extra_at = ifd_at + (8 if big else 2) + esize * len(entries) + (8 if big else 4)
    ifd, extra = bytearray(), bytearray()
    ifd += struct.pack(bo + ("Q" if big else "H"), len(entries))
    for tag, typ, vals in entries:
        raw = struct.pack(bo + code[typ] * len(vals), *vals)
        if len(raw) <= inline:
            field = raw.ljust(inline, b"\0")
        else:
            field = struct.pack(bo + ("Q" if big else "I"), extra_at + len(extra))
            extra += raw
        ifd += struct.pack(bo + ("HHQ" if big else "HHI"), tag, typ, len(vals)) + field
    ifd += b"\0" * (8 if big else 4)
    mark = b"II" if bo == "<" else b"MM"
    header = mark + (struct.pack(bo + "HHHQ", 43, 8, 0, ifd_at) if big
                     else struct.pack(bo + "HI", 42, ifd_at))
    with open(path, "wb") as fh:
        fh.write(header + b"".join(chunks) + bytes(ifd) + bytes(extra))


@pytest.mark.parametrize("layout", [
    dict(tile=(16, 16)), dict(tile=(32, 16), deflate=True), dict(rows_per_strip=7),
    dict(rows_per_strip=5, deflate=True, bo=">"), dict(tile=(16, 32), bo=">", big=True),
    dict(rows_per_strip=9, big=True, deflate=True)])
@pytest.mark.parametrize("dtype", [np.float32, np.float64, np.int16])
def test_tiles_strips_byte_orders_and_bigtiff(tmp_path, layout, dtype):
    a = (np.random.default_rng(5).normal(size=(45, 37)) * 1000).astype(dtype)
    p = str(tmp_path / "t.tif")
    _write_tiff(p, a, **layout)
    got, meta = read_geotiff(p)
    assert got.dtype == np.dtype(dtype) and got.shape == (45, 37)
    np.testing.assert_array_equal(got, a)


@pytest.mark.parametrize("planar", [1, 2])
def test_multiband_reads_the_requested_band(tmp_path, planar):
    a = np.random.default_rng(6).normal(size=(20, 24, 3)).astype(np.float32)
    p = str(tmp_path / "b.tif")
    _write_tiff(p, a, planar=planar, rows_per_strip=6, deflate=True)
    for band in (1, 2, 3):
        got, meta = read_geotiff(p, band=band)
        np.testing.assert_array_equal(got, a[:, :, band - 1])
    assert meta["count"] == 3
    with pytest.raises(ValueError):
        read_geotiff(p, band=4)


def test_rejects_non_tiff(tmp_path):
    p = tmp_path / "x.tif"
    p.write_bytes(b"not a tiff at all")
    with pytest.raises(ValueError):
        read_geotiff(str(p))
