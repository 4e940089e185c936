"""Result rasters with the reference's post-processing call, without rasterio.

`exportRaster_tiff(DEM_path, outPutPath)` keeps the reference's signature and
output (HP/postProcessing.py:26-196): every exported field file in outPutPath
(`<field>_<str(t)>.pt`, a compacted vector of the DEM's valid cells, as
`FusedSolver.export_fields` and `Godunov.exportField` write them) is
scattered into the DEM's raster, the no-data cells get -9999, and the raster
is written as a float32 GeoTIFF with the DEM's transform and CRS (its EPSG
code, or its GeoKey tags copied verbatim when the CRS is not one EPSG code)
under the reference's name (`<prefix>_<time>tif`).
"""
from __future__ import annotations

import numpy as np

from .geotiff import export_raster_tiff, read_geotiff


def exportRaster_tiff(DEM_path: str, outPutPath: str) -> list[str]:
    """GeoTIFFs of the exported field files of outPutPath on the DEM's grid;
    returns the paths written."""
    dem, meta = read_geotiff(DEM_path, masked=True)
    valid = ~np.ma.getmaskarray(dem)
    epsg, geokeys = None, None
    if meta["crs"] and meta["crs"].startswith("EPSG:"):
        epsg = int(meta["crs"][5:])
    elif meta.get("geokeys"):
        # a CRS that is not one EPSG code: the DEM's GeoKey tags, verbatim
        geokeys = meta["geokeys"]
    return export_raster_tiff(outPutPath, valid.astype(np.int32), transform=meta["transform"],
                              epsg=epsg, nodata=-9999.0, pattern="*.pt", geokeys=geokeys)
