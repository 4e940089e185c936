"""Seeded synthetic inputs of the benchmark configurations.

No public dataset is involved: every case is generated here from a seed with
the shapes, sizes and value ranges of the workload it stands for.

  dam_break        256 x 256, 1 m cells, flat bed, h = 1 m for x < 128 and
                   0.01 m elsewhere, n = 0.03, reflective walls, CFL 0.5
  urban_catchment  n x n (2048 in the headline case), 2 m cells, DEM = seeded
                   Gaussian random field with k^-3 spectrum scaled to 0-50 m
                   plus 8 % of cells raised 10 m as 5-30-cell rectangles;
                   30 % "road" zone n = 0.035, other cells n = 0.08; open ring;
                   dry start; uniform rain 50 mm/h for 3600 s
  ensemble         catchments with sides drawn from 256-1536 cells, each with
                   its own double-triangle hyetograph (peaks 20-120 mm/h)
  adjoint_case     n x n (1024 in the headline case) DEM as urban_catchment,
                   16 Voronoi Manning zones from seeded sites with n drawn
                   from U(0.02, 0.10), 32 gauges on random valid cells,
                   rain 50 mm/h, optional initial pond
  coupled_case     n x n (8192 in the headline case), 1 m cells, DEM as
                   urban_catchment, rain 100 mm/h for 1800 s, Q_GIVEN inflow on
                   the west edge (hydrograph 0 -> 500 -> 0 m^3/s over 1800 s as
                   unit discharge sampled every 10 s), open elsewhere, and
                   agent cells drawn uniformly over non-building cells
  channel          the 25 x 225 back-channel case: H_GIVEN inflow, OPEN
                   outflow, walls (HP/backCase.ipynb scenario, own geometry)

Rasters carry a one-cell no-data ring (mask -9999), as the reference's
``roll``-based neighbour table requires.
"""
from __future__ import annotations

import math

import numpy as np

from .fused import Catchment
from .topology import boundary_codes

MM_PER_H = 1.0e-3 / 3600.0  # m/s per mm/h


def _ring(n_rows: int, n_cols: int) -> np.ndarray:
    nodata = np.zeros((n_rows + 2, n_cols + 2), dtype=bool)
    nodata[0, :] = nodata[-1, :] = True
    nodata[:, 0] = nodata[:, -1] = True
    return nodata


def gaussian_field(n_rows: int, n_cols: int, seed: int, slope: float = 3.0) -> np.ndarray:
    """Zero-mean random field whose power spectrum falls as k^-slope."""
    rng = np.random.default_rng(seed)
    noise = rng.standard_normal((n_rows, n_cols))
    ky = np.fft.fftfreq(n_rows)[:, None]
    kx = np.fft.rfftfreq(n_cols)[None, :]
    k = np.sqrt(kx * kx + ky * ky)
    k[0, 0] = 1.0
    amp = k ** (-slope / 2.0)
    amp[0, 0] = 0.0
    f = np.fft.irfft2(np.fft.rfft2(noise) * amp, s=(n_rows, n_cols))
    return f


def urban_dem(n_rows: int, n_cols: int, seed: int, relief: float = 50.0,
              building_frac: float = 0.08, building_h: float = 10.0) -> tuple[np.ndarray, np.ndarray]:
    """DEM in [0, relief] + raised rectangles; returns (z, building mask)."""
    f = gaussian_field(n_rows, n_cols, seed)
    f = (f - f.min()) / max(f.max() - f.min(), 1e-12) * relief
    rng = np.random.default_rng(seed + 7919)
    bmask = np.zeros((n_rows, n_cols), dtype=bool)
    target = building_frac * n_rows * n_cols
    covered = 0
    while covered < target:
        hgt = int(rng.integers(5, 31))
        wid = int(rng.integers(5, 31))
        r0 = int(rng.integers(0, max(n_rows - hgt, 1)))
        c0 = int(rng.integers(0, max(n_cols - wid, 1)))
        blk = bmask[r0:r0 + hgt, c0:c0 + wid]
        covered += int((~blk).sum())
        blk[:] = True
    return f + building_h * bmask, bmask


def road_mask(n_rows: int, n_cols: int, seed: int, frac: float = 0.30) -> np.ndarray:
    f = gaussian_field(n_rows, n_cols, seed + 104729, slope=4.0)
    thr = np.quantile(f, frac)
    return f <= thr


def dam_break(n: int = 256, ring_code: int = 40, manning: float = 0.03) -> dict:
    """Config 1 rasters (reference argument layout) plus solver settings."""
    nodata = _ring(n, n)
    mask = boundary_codes(nodata, default_bc=ring_code)
    z = np.zeros(mask.shape)
    h = np.zeros(mask.shape)
    cols = np.arange(mask.shape[1]) - 1  # valid column index
    h[:, :] = np.where(cols[None, :] < n // 2, 1.0, 0.01)
    h[nodata] = 0.0
    zeros = np.zeros(mask.shape)
    return dict(mask=mask, z=z, h=h, qx=zeros.copy(), qy=zeros.copy(), wl=z + h,
                landuse=np.zeros(mask.shape, dtype=np.uint8), manning=[manning], dx=1.0,
                cfl=0.5, first_dt=1.0e-4, second_order=True, steps=1000)


def urban_catchment(n: int = 2048, dx: float = 2.0, seed: int = 0, rain_mm_h: float = 50.0,
                    duration: float = 3600.0, n_rows: int | None = None) -> dict:
    """Config 2 rasters and settings (single instance); n_rows x n valid cells
    when n_rows is given (default square)."""
    m = n if n_rows is None else n_rows
    nodata = _ring(m, n)
    mask = boundary_codes(nodata, default_bc=50)
    z = np.zeros(mask.shape)
    zi, bmask = urban_dem(m, n, seed)
    z[1:-1, 1:-1] = zi
    zone = np.ones(mask.shape, dtype=np.uint8)
    zone[1:-1, 1:-1] = np.where(road_mask(m, n, seed), 0, 1)
    zeros = np.zeros(mask.shape)
    rate = rain_mm_h * MM_PER_H
    return dict(mask=mask, z=z, h=zeros.copy(), qx=zeros.copy(), qy=zeros.copy(), wl=z.copy(),
                landuse=zone, manning=[0.035, 0.08], dx=dx, cfl=0.5, first_dt=1.0e-4,
                rain=np.array([[0.0, rate], [duration, rate]]), t_end=duration,
                buildings=bmask)


def double_triangle_hyetograph(seed: int, duration: float = 3600.0) -> np.ndarray:
    """Two triangular peaks of U(20, 120) mm/h at U(0, 1800) s, [T, 2] in m/s."""
    rng = np.random.default_rng(seed)
    peaks = np.sort(rng.uniform(0.0, 1800.0, 2))
    amps = rng.uniform(20.0, 120.0, 2) * MM_PER_H
    width = 600.0
    times = np.linspace(0.0, duration, 121)
    rate = np.zeros_like(times)
    for p, a in zip(peaks, amps):
        rate = np.maximum(rate, a * np.clip(1.0 - np.abs(times - p) / width, 0.0, None))
    return np.stack([times, rate], axis=1)


def catchment_from(d: dict, **over) -> Catchment:
    kw = dict(mask=d["mask"], z=d["z"], h=d["h"], qx=d.get("qx"), qy=d.get("qy"),
              zone=d.get("landuse"), manning=d["manning"], dx=d["dx"], cfl=d["cfl"],
              dt0=d["first_dt"], rain=d.get("rain"), given_depth=d.get("given_depth"),
              given_wl=d.get("given_wl"), given_q=d.get("given_q"),
              t_end=d.get("t_end", math.inf))
    kw.update(over)
    return Catchment(**kw)


def ensemble(count: int = 64, seed: int = 0, lo: int = 256, hi: int = 1536,
             dx: float = 2.0) -> list[dict]:
    rng = np.random.default_rng(seed)
    sides = rng.integers(lo, hi + 1, size=count)
    out = []
    for k, s in enumerate(sides):
        d = urban_catchment(int(s), dx=dx, seed=seed * 1000 + k)
        d["rain"] = double_triangle_hyetograph(seed * 1000 + k)
        out.append(d)
    return out


def channel(n_rows: int = 25, n_cols: int = 225, dx: float = 0.2012, inflow_h: float = 0.242,
            manning: float = 0.01, wall_code: int = 40) -> dict:
    """Back-channel case: H_GIVEN (60) left, OPEN (50) right, walls top/bottom."""
    mask = np.full((n_rows + 2, n_cols + 2), 10, dtype=np.int32)
    mask[1, :] = wall_code
    mask[-2, :] = wall_code
    mask[:, 1] = 60
    mask[:, -2] = 50
    mask[0, :] = mask[-1, :] = -9999
    mask[:, 0] = mask[:, -1] = -9999
    zeros = np.zeros(mask.shape)
    return dict(mask=mask, z=zeros.copy(), h=zeros.copy(), qx=zeros.copy(), qy=zeros.copy(),
                wl=zeros.copy(), landuse=np.zeros(mask.shape, dtype=np.uint8),
                manning=[manning], dx=dx, cfl=0.5, first_dt=1.0e-3,
                given_depth=np.array([[0.0, inflow_h], [600.0, inflow_h]]),
                given_q=np.array([[0.0, 0.202, 0.0], [600.0, 0.202, 0.0]]),
                rain=np.array([[0.0, 0.0], [200.0, 0.0]]), t_end=8.0)


def voronoi_zones(n_rows: int, n_cols: int, n_zones: int, seed: int) -> np.ndarray:
    """Zone of every cell: index of the nearest of n_zones seeded sites."""
    rng = np.random.default_rng(seed)
    sites = rng.uniform(0.0, 1.0, (n_zones, 2)) * np.array([n_rows, n_cols])
    zone = np.empty((n_rows, n_cols), dtype=np.uint8)
    cc = np.arange(n_cols, dtype=np.float64)
    for r in range(n_rows):
        d = (r - sites[:, 0:1]) ** 2 + (cc[None, :] - sites[:, 1:2]) ** 2
        zone[r] = np.argmin(d, axis=0)
    return zone


def adjoint_case(n: int = 1024, dx: float = 2.0, seed: int = 0, n_zones: int = 16,
                 n_gauges: int = 32, rain_mm_h: float = 50.0, pond: float = 0.0,
                 relief: float = 50.0) -> dict:
    """Manning-calibration case: DEM as urban_catchment, Voronoi zones with
    true n ~ U(0.02, 0.10), gauges on random valid cells.  pond > 0 adds an
    initial water level pond m above the lowest quarter of the bed."""
    d = urban_catchment(n, dx=dx, seed=seed, rain_mm_h=rain_mm_h)
    if relief != 50.0:
        zi, _ = urban_dem(n, n, seed, relief=relief)
        d["z"][1:-1, 1:-1] = zi
    rng = np.random.default_rng(seed + 104729)
    zone = np.zeros(d["mask"].shape, dtype=np.uint8)
    zone[1:-1, 1:-1] = voronoi_zones(n, n, n_zones, seed + 31)
    d["landuse"] = zone
    d["manning"] = list(rng.uniform(0.02, 0.10, n_zones))
    valid = d["mask"] > 0
    if pond > 0.0:
        zin = d["z"][valid]
        level = np.quantile(zin, 0.25) + pond
        d["h"] = np.where(valid, np.maximum(level - d["z"], 0.0), 0.0)
    rr, cc = np.nonzero(valid)
    pick = rng.choice(rr.size, size=n_gauges, replace=False)
    d["gauge_rows"], d["gauge_cols"] = rr[pick], cc[pick]
    return d


def coupled_case(n: int = 8192, dx: float = 1.0, seed: int = 0, agents: int = 100_000,
                 peak_q: float = 500.0, duration: float = 1800.0) -> dict:
    """Coupled-run rasters: urban DEM, 100 mm/h rain, a Q_GIVEN inflow edge
    (west) with a triangular hydrograph peaking at peak_q m^3/s at duration/2,
    given as unit discharge q = Q / (n dx) every 10 s, and `agents` agent cells
    (row-major order, as the reference reports them) on non-building cells."""
    d = urban_catchment(n, dx=dx, seed=seed, rain_mm_h=100.0, duration=duration)
    nodata = _ring(n, n)
    d["mask"] = boundary_codes(nodata, default_bc=50, boxes=[(1, n + 1, 1, 2, 7)])
    t = np.arange(0.0, duration + 10.0, 10.0)
    Q = peak_q * np.clip(1.0 - np.abs(t - duration / 2) / (duration / 2), 0.0, None)
    d["given_q"] = np.stack([t, Q / (n * dx), np.zeros_like(t)], axis=1)
    ok = np.zeros(d["mask"].shape, dtype=bool)
    ok[1:-1, 1:-1] = ~d["buildings"]
    rr, cc = np.nonzero(ok)
    rng = np.random.default_rng(seed + 65537)
    pick = np.sort(rng.choice(rr.size, size=min(agents, rr.size), replace=False))
    d["agent_rows"], d["agent_cols"] = rr[pick], cc[pick]
    return d
