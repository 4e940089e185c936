"""GeoTIFF output (the reference's exportRaster_tiff, HP/postProcessing.py:26-196,
without rasterio): pixels and tags read back with Pillow, and the reference's
naming and scatter of exported field files."""
import numpy as np
import pytest
import torch
from PIL import Image

from hipims_b200.geotiff import export_raster_tiff, reference_tif_name, write_geotiff


def _read(path):
    im = Image.open(path)
    assert im.mode == "F"
    return np.array(im), dict(im.tag_v2)


def test_write_geotiff_pixels_and_georeferencing(tmp_path):
    rng = np.random.default_rng(1)
    a = rng.normal(size=(37, 53)).astype(np.float32)
    a[3, 4] = -9999.0
    p = write_geotiff(str(tmp_path / "a.tif"), a, transform=(2.0, 0.0, 500000.0, 0.0, -2.0,
                                                            4200000.0), epsg=27700)
    got, tags = _read(p)
    np.testing.assert_array_equal(got, a)
    one = lambda v: v[0] if isinstance(v, tuple) else v
    assert one(tags[339]) == 3 and one(tags[258]) == 32             # IEEE float, 32 bits
    assert tuple(tags[33550]) == (2.0, 2.0, 0.0)                    # pixel scale
    assert tuple(tags[33922]) == (0.0, 0.0, 0.0, 500000.0, 4200000.0, 0.0)  # tie point
    keys = list(tags[34735])
    assert keys[:4] == [1, 1, 0, 3]
    entries = {keys[i]: keys[i + 3] for i in range(4, len(keys), 4)}
    assert entries == {1024: 1, 1025: 1, 3072: 27700}               # projected, EPSG:27700
    assert tags[42113] == "-9999"


def test_write_geotiff_rotated_and_geographic(tmp_path):
    a = np.arange(12, dtype=np.float64).reshape(3, 4)
    p = write_geotiff(str(tmp_path / "r.tif"), a, transform=(1.0, 0.5, 10.0, 0.25, -1.0, 20.0),
                      epsg=4326, nodata=None)
    got, tags = _read(p)
    np.testing.assert_array_equal(got, a.astype(np.float32))
    assert 33550 not in tags and 42113 not in tags
    m = tuple(tags[34264])
    assert m[:8] == (1.0, 0.5, 0.0, 10.0, 0.25, -1.0, 0.0, 20.0) and m[15] == 1.0
    keys = list(tags[34735])
    entries = {keys[i]: keys[i + 3] for i in range(4, len(keys), 4)}
    assert entries == {1024: 2, 1025: 1, 2048: 4326}                # geographic, EPSG:4326


def test_reference_tif_names():
    assert reference_tif_name("out/h_tensor([3600.], device='cuda:0', dtype=torch.float64).pt") \
        == "out/h_3600.tif"
    assert reference_tif_name("out/h_max_tensor([60.], device='cuda:0').pt") == "out/h_max_60.tif"
    # a fractional time keeps the reference's missing dot
    assert reference_tif_name("out/qx_tensor([12.5000], device='cuda:0').pt") == \
        "out/qx_12.5000tif"


def test_export_raster_tiff_scatters_compacted_fields(tmp_path):
    mask = np.full((6, 7), -9999, dtype=np.int32)
    mask[1:-1, 1:-1] = 10
    mask[2, 3] = -9999                                              # an interior hole
    valid = mask > 0
    vec = torch.arange(int(valid.sum()), dtype=torch.float64) * 0.5
    name = "h_tensor([3600.], device='cuda:0', dtype=torch.float64).pt"
    torch.save(vec, str(tmp_path / name))
    paths = export_raster_tiff(str(tmp_path), mask, transform=(1.0, 0, 0, 0, -1.0, 6.0),
                               epsg=32630)
    assert paths == [str(tmp_path / "h_3600.tif")]
    got, _ = _read(paths[0])
    want = np.full(mask.shape, -9999.0, dtype=np.float32)
    want[valid] = vec.numpy()
    np.testing.assert_array_equal(got, want)
    with pytest.raises(ValueError):
        torch.save(vec[:-1], str(tmp_path / name))
        export_raster_tiff(str(tmp_path), mask)


def test_export_keeps_a_crs_that_is_not_an_epsg_code(tmp_path):
    """A DEM whose CRS is user-defined (ProjectedCSType 32767, parameters in
    GeoDoubleParams, a citation in GeoAsciiParams): exportRaster_tiff copies
    the DEM's GeoKey tags into every result raster instead of dropping them."""
    from hipims_b200.geotiff import read_geotiff
    from hipims_b200.postprocessing import exportRaster_tiff

    geokeys = {
        # version 1.1.0, 5 keys: model projected, pixel is area, user-defined
        # projected CRS, its citation (ascii params 0..), a linear unit (m)
        34735: [1, 1, 0, 5, 1024, 0, 1, 1, 1025, 0, 1, 1, 3072, 0, 1, 32767,
                3073, 34737, 24, 0, 3076, 0, 1, 9001],
        34736: [6378137.0, 298.257223563, 0.9996, 500000.0],
        34737: "custom transverse merc|",
    }
    dem = np.full((5, 6), -9999.0)
    dem[1:-1, 1:-1] = 3.0
    dem_path = write_geotiff(str(tmp_path / "dem.tif"), dem,
                             transform=(2.0, 0.0, 1000.0, 0.0, -2.0, 5000.0), geokeys=geokeys)
    _, meta = read_geotiff(dem_path)
    assert meta["crs"] is None and meta["geokeys"][34735] == geokeys[34735]
    out = tmp_path / "out"
    out.mkdir()
    vec = torch.arange(12, dtype=torch.float64)
    torch.save(vec, str(out / "h_tensor([60.], device='cuda:0', dtype=torch.float64).pt"))
    paths = exportRaster_tiff(dem_path, str(out))
    assert paths == [str(out / "h_60.tif")]
    got, tags = _read(paths[0])
    assert list(tags[34735]) == geokeys[34735]
    assert tuple(tags[34736]) == tuple(geokeys[34736])
    assert tags[34737] == geokeys[34737]
    assert tuple(tags[33550]) == (2.0, 2.0, 0.0)
    want = np.full(dem.shape, -9999.0, dtype=np.float32)
    want[1:-1, 1:-1] = vec.numpy().reshape(3, 4)
    np.testing.assert_array_equal(got, want)
