"""Raster inputs with the reference's pre-processing interface
(hipims_b200.preprocessing, HP/preProcessing.py:140-390) on GeoTIFFs written
here: boundary coding from boxes in map units against the raster-index
coding of hipims_b200.topology, gauge indices, land-use renumbering and the
rain-station mask."""
import numpy as np
import pytest
import torch

from hipims_b200 import preprocessing as P
from hipims_b200.geotiff import write_geotiff
from hipims_b200.topology import boundary_codes

# 2 m cells, upper-left corner at (1000, 5000)
T = (2.0, 0.0, 1000.0, 0.0, -2.0, 5000.0)


def _dem(tmp_path, ny=30, nx=40, seed=0):
    rng = np.random.default_rng(seed)
    z = rng.uniform(10.0, 20.0, size=(ny, nx)).astype(np.float32)
    nodata = np.zeros((ny, nx), dtype=bool)
    nodata[0, :] = nodata[-1, :] = nodata[:, 0] = nodata[:, -1] = True
    nodata[:6, :9] = True           # a notch in the corner
    nodata[14:17, 20:23] = True     # an interior hole
    z[nodata] = -9999.0
    path = write_geotiff(str(tmp_path / "dem.tif"), z, transform=T, epsg=27700)
    return path, z, nodata


def _xy(row, col):
    """Map position of the pixel centre."""
    return T[2] + (col + 0.5) * T[0], T[5] + (row + 0.5) * T[4]


def _box(r0, r1, c0, c1):
    """Map box (left, bottom, right, top) of raster rows [r0, r1) and columns [c0, c1)."""
    return [T[2] + c0 * T[0], T[5] + r1 * T[4], T[2] + c1 * T[0], T[5] + r0 * T[4]]


def test_rowcol_floors_like_rasterio():
    r, c = P.rowcol(T, [1000.0, 1001.9, 1002.0, 1079.99], [5000.0, 4998.1, 4998.0, 4940.01])
    assert r.tolist() == [0, 0, 1, 29] and c.tolist() == [0, 0, 1, 39]


def test_dem_and_boundary_coding_match_the_raster_index_coding(tmp_path):
    path, z, nodata = _dem(tmp_path)
    boxes_rc = [(0, 30, 0, 3, 6), (0, 30, 37, 40, 5), (25, 30, 9, 30, 7), (0, 3, 9, 40, 3),
                (20, 30, 0, 2, 6)]
    # the last box reaches past the raster's left and bottom edges: clipped
    # to its bounds, it covers rows 20-29 of columns 0-1
    world = [_box(*b[:4]) for b in boxes_rc[:-1]] + [[900.0, 4900.0, 1004.0, 4960.0]]
    dem, mask, meta, gauges = P.importDEMData_And_BC(
        path, "cpu", boundBox=np.array(world), default_BC=40, bc_type=[b[4] for b in boxes_rc])
    want = boundary_codes(nodata, default_bc=40, boxes=boxes_rc)
    want[want < 0] = 0
    assert mask.dtype == torch.int32
    np.testing.assert_array_equal(mask.numpy(), want)
    assert set(np.unique(want)) >= {0, 1, 40, 60, 61, 50, 70, 30}
    np.testing.assert_array_equal(dem.numpy(), z)
    assert meta["transform"] == T and meta["crs"] == "EPSG:27700"
    assert gauges.numel() == 0


def test_boundary_type_names_and_fall(tmp_path):
    path, _, nodata = _dem(tmp_path)
    names = ["H_GIVEN", "FALL"]
    _, mask, _, _ = P.importDEMData_And_BC(path, "cpu", boundBox=np.array(
        [_box(0, 30, 0, 3), _box(25, 30, 9, 30)]), default_BC=50, bc_type=names)
    want = boundary_codes(nodata, default_bc=50, boxes=[(0, 30, 0, 3, 6), (25, 30, 9, 30, 9)])
    want[want < 0] = 0
    np.testing.assert_array_equal(mask.numpy(), want)
    with pytest.raises(ValueError):
        P.importDEMData_And_BC(path, "cpu", boundBox=np.array([_box(0, 30, 0, 3)]),
                               bc_type=["NOT_A_TYPE"])


def test_gauges_map_to_compacted_indices_in_the_given_order(tmp_path):
    path, _, nodata = _dem(tmp_path)
    cells = [(20, 30), (7, 10), (28, 38), (10, 25)]
    pos = np.array([_xy(r, c) for r, c in cells])
    _, _, _, g = P.importDEMData_And_BC(path, "cpu", gauges_position=pos)
    compact = -np.ones(nodata.shape, dtype=np.int64)
    compact[~nodata] = np.arange(int((~nodata).sum()))
    assert g.dtype == torch.int64
    assert g.tolist() == [int(compact[r, c]) for r, c in cells]


def test_import_dem_data(tmp_path):
    path, z, nodata = _dem(tmp_path)
    dem, valid, ring, meta = P.importDEMData(path, "cpu")
    np.testing.assert_array_equal(valid.numpy(), ~nodata)
    codes = boundary_codes(nodata, default_bc=50)
    np.testing.assert_array_equal(ring.numpy(), codes == 50)
    np.testing.assert_array_equal(dem.numpy(), z)


def test_landuse_renumbering(tmp_path):
    codes = np.array([[3, 3, 7], [9, 255, 7], [3, 9, 9]], dtype=np.uint8)
    p = write_geotiff(str(tmp_path / "lu.tif"), codes.astype(np.float32), transform=T,
                      nodata=255.0)
    lu, idx = P.importLanduseData(p, "cpu")
    # no-data -> 1; unique [1, 3, 7, 9]: 3 -> 0, 7 -> 1, 9 -> 2, 1 stays 1
    assert lu.numpy().tolist() == [[0, 0, 1], [2, 1, 1], [0, 2, 2]]
    assert idx.tolist() == [0, 1, 2]
    lu1, idx1 = P.importLanduseData(p, "cpu", level=1)
    # int(c / 10) - 1 with no-data -> 11
    assert lu1.numpy().tolist() == [[-1, -1, -1], [-1, 0, -1], [-1, -1, -1]]
    assert idx1.tolist() == [0]


def test_rain_station_mask(tmp_path):
    m = np.array([[0, 1, 2], [2, -9999, 1]], dtype=np.float32)
    p = write_geotiff(str(tmp_path / "rain.tif"), m, transform=T)
    r = P.importRainStationMask(p, "cpu")
    assert r.dtype == torch.int16
    assert r.numpy().tolist() == [[0, 1, 2], [2, 0, 1]]


def test_imported_rasters_drive_the_oracle_like_the_raster_index_coding(tmp_path):
    """A run set up from the imported DEM and mask (0 on no-data, as the
    reference's) takes the same steps as one set up with the -9999 coding of
    hipims_b200.topology."""
    from oracle import oracle as O

    path, z, nodata = _dem(tmp_path)
    dem, mask, _, _ = P.importDEMData_And_BC(path, "cpu", boundBox=np.array(
        [_box(0, 30, 0, 3)]), default_BC=30, bc_type=[6])
    h = np.where(nodata, 0.0, np.linspace(0.0, 0.5, z.shape[1])[None, :] * (z > 15))
    base = dict(z=dem.numpy().astype(np.float64), h=h, qx=np.zeros_like(h), qy=np.zeros_like(h),
                manning=[0.03], dx=2.0, cfl=0.5, first_dt=1e-3,
                given_depth=np.array([[0.0, 0.2], [100.0, 0.2]]))
    codes = boundary_codes(nodata, default_bc=30, boxes=[(0, 30, 0, 3, 6)])
    a = O.Sim(dict(base, mask=mask.numpy()), order=2)
    b = O.Sim(dict(base, mask=codes), order=2)
    a.run(20)
    b.run(20)
    sa, sb = a.state(), b.state()
    assert sa["t"] == sb["t"] and np.isfinite(sa["h"]).all()
    for f in ("h", "qx", "qy"):
        np.testing.assert_array_equal(sa[f], sb[f])


def test_export_raster_tiff_on_the_dem_grid(tmp_path):
    """exportRaster_tiff(DEM_path, outPutPath) as HP/postProcessing.py:26-196:
    each exported field file goes to the DEM's valid cells, -9999 elsewhere,
    with the DEM's georeferencing, under the reference's name."""
    from hipims_b200.geotiff import read_geotiff
    from hipims_b200.postprocessing import exportRaster_tiff

    path, _, nodata = _dem(tmp_path)
    out = tmp_path / "out"
    out.mkdir()
    n = int((~nodata).sum())
    vec = torch.arange(n, dtype=torch.float64) * 0.01
    torch.save(vec, str(out / "h_tensor([3600.], device='cuda:0').pt"))
    torch.save(-vec, str(out / "qx_tensor([3600.], device='cuda:0').pt"))
    written = sorted(exportRaster_tiff(path, str(out)))
    assert [p.rsplit("/", 1)[1] for p in written] == ["h_3600.tif", "qx_3600.tif"]
    r, meta = read_geotiff(str(out / "h_3600.tif"))
    assert r.dtype == np.float32 and meta["transform"] == T and meta["crs"] == "EPSG:27700"
    assert meta["nodata"] == -9999.0
    np.testing.assert_array_equal(r[~nodata], vec.numpy().astype(np.float32))
    assert (r[nodata] == -9999.0).all()
