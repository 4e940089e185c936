"""Host-side logic that needs no GPU: topology, boundary coding, scenario
generators, rain interpolation, the dense layout builder."""
import numpy as np
import pytest
import torch

from hipims_b200 import _lib, scenarios as S, topology as T
from hipims_b200.fused import _Instance
from oracle import oracle as O


@pytest.mark.parametrize("code", [1, 10, 30, 40, 50, 51, 60, 61, 72, 80, 512, 9])
def test_decode_bc_matches_oracle(code):
    assert T.decode_bc(code) == O.decode_bc(code)


def test_compact_index_matches_oracle():
    rng = np.random.default_rng(0)
    nodata = rng.uniform(size=(17, 23)) < 0.2
    nodata[0, :] = nodata[-1, :] = nodata[:, 0] = nodata[:, -1] = True
    mask = T.boundary_codes(nodata, default_bc=50, boxes=[(0, 17, 0, 8, 6)])
    idx = T.compact_index(torch.as_tensor(mask)).numpy()
    np.testing.assert_array_equal(idx, O.build_index(mask))


def test_compact_index_wraps_like_roll():
    mask = np.ones((4, 5), dtype=np.int32)
    idx = T.compact_index(torch.as_tensor(mask)).numpy().reshape(5, -1)
    # cell (0, 4): east neighbour wraps to (0, 0) = id 0, north wraps to (3, 4) = id 19
    assert idx[1, 4] == 0 and idx[2, 4] == 19


def test_boundary_codes_ring_and_boxes():
    nodata = np.zeros((6, 8), dtype=bool)
    nodata[0, :] = nodata[-1, :] = nodata[:, 0] = nodata[:, -1] = True
    m = T.boundary_codes(nodata, default_bc=50, boxes=[(0, 6, 0, 2, 6), (0, 6, 6, 8, 6)])
    assert m[0, 0] == -9999 and m[2, 3] == 1
    assert m[2, 1] == 60 and m[2, 6] == 61 and m[1, 3] == 50


def test_urban_dem_statistics():
    z, b = S.urban_dem(256, 256, seed=5)
    base = z - 10.0 * b
    assert base.min() >= -1e-9 and base.max() <= 50.0 + 1e-9
    assert 0.08 <= b.mean() < 0.10
    r = S.road_mask(256, 256, seed=5)
    assert abs(r.mean() - 0.30) < 0.01
    z2, _ = S.urban_dem(256, 256, seed=5)
    np.testing.assert_array_equal(z, z2)


def test_hyetograph_shape():
    h = S.double_triangle_hyetograph(3)
    assert h[0, 0] == 0.0 and h[-1, 0] == 3600.0
    peak = h[:, 1].max() / S.MM_PER_H
    assert 20.0 <= peak <= 120.0 + 1e-9


def test_dense_layout_builder():
    d = S.dam_break(40)
    c = S.catchment_from(d)
    ins = _Instance(c, torch.float32, "cpu", (32, 32))
    assert ins.pitch % 32 == 0 and ins.code_pitch % 128 == 0
    assert ins.rows_s >= 64 + 4 and ins.tiles_x == 2 and ins.tiles_y == 2
    code = ins.code.numpy()
    PY, CPX = _lib.HB_PAD_Y, _lib.HB_CODE_PAD_X
    assert code[0, 0] >> 4 == _lib.HB_NODATA_CLASS
    r = code[PY:PY + 42, CPX:CPX + 42]
    assert (r[0] >> 4 == _lib.HB_NODATA_CLASS).all()
    assert ins.bc_type[r[1, 1] >> 4] == 4 and ins.bc_type[r[5, 5] >> 4] == 1
    h = ins.raster(ins.h[0]).numpy()
    np.testing.assert_array_equal(h, np.where(d["mask"] > 0, d["h"], 0.0).astype(np.float32))
    assert ins.bug == (1, 1)


def test_datum_keeps_bed_exact():
    d = S.urban_catchment(100, seed=1)
    c = S.catchment_from(d)
    ins = _Instance(c, torch.float32, "cpu", (32, 32))
    zrel = ins.raster(ins.z).double().numpy()
    zabs = zrel + ins.z_abs_offset
    v = d["mask"] > 0
    assert np.abs(zabs[v] - d["z"][v]).max() < 1e-5
    # each cell sits between its block's datum (floor of the block minimum)
    # and the block maximum
    for by in range(ins.datum_np.shape[0]):
        for bx in range(ins.datum_np.shape[1]):
            sl = (slice(by * 64, (by + 1) * 64), slice(bx * 64, (bx + 1) * 64))
            zb, vb = d["z"][sl][v[sl]], zrel[sl][v[sl]]
            if zb.size:
                assert vb.min() >= 0.0 and vb.max() <= zb.max() - zb.min() + 1.0
    assert (ins.datum_np == np.floor(ins.datum_np)).all()


def test_rain_interpolation_matches_oracle_cursor():
    from hipims_b200.solver import Godunov

    R = np.array([[0.0, 1.0, 2.0], [10.0, 3.0, 0.0], [30.0, 0.0, 1.0]])
    g = Godunov("cpu", 1.0, 0.5, 100.0)
    for t, want in ((0.0, [1.0, 2.0]), (5.0, [2.0, 1.0]), (20.0, [1.5, 0.5]), (30.0, [0, 0])):
        g.t = torch.tensor([t], dtype=torch.float64)
        np.testing.assert_allclose(g._interp_rain(R), want)


def _brute_grid_cost(valid, tile, origin, bug):
    """tile_grid_cost restated tile by tile."""
    ty, tx = tile
    sy, sx = origin
    rows, cols = valid.shape
    pv = np.zeros((rows + sy + ty + 8, cols + sx + tx + 16), dtype=bool)
    pv[4 + sy:4 + sy + rows, 8 + sx:8 + sx + cols] = valid  # kernel raster at (4, 8)
    kb = None if bug is None else (bug[0] + sy, bug[1] + sx)
    total = 0.0
    for a in range((rows + sy + ty - 1) // ty):
        for b in range((cols + sx + tx - 1) // tx):
            y0, x0 = a * ty, b * tx
            box = pv[4 + y0 - 2:4 + y0 + ty + 2, 8 + x0 - 4:8 + x0 + tx + 4]
            allv = box.all() and not (kb is not None and y0 - 2 <= kb[0] < y0 + ty + 2
                                      and x0 - 4 <= kb[1] < x0 + tx + 4)
            live = [i for i in range(ty) if pv[4 + y0 + i, 8 + x0:8 + x0 + tx].any()]
            if allv:
                total += 1.0
            elif not live:
                total += 0.1
            else:
                span = live[-1] + 1 - live[0]
                total += 0.4 + 1.1 * (-(-span // 4)) / (ty / 4)
    return total


def test_tile_grid_cost_matches_tile_by_tile_count():
    from hipims_b200.fused import _first_valid_cell, tile_grid_cost

    rng = np.random.default_rng(3)
    for n, m in ((130, 150), (97, 200)):
        nodata = np.zeros((n, m), dtype=bool)
        nodata[0, :] = nodata[-1, :] = nodata[:, 0] = nodata[:, -1] = True
        nodata |= rng.uniform(size=(n, m)) < 0.002
        mask = T.boundary_codes(nodata, default_bc=50)
        valid = mask > 0
        bug = _first_valid_cell(mask)
        for origin in ((0, 0), (7, 63), (3, 17), (31, 1)):
            assert tile_grid_cost(valid, (32, 64), origin, bug) == \
                pytest.approx(_brute_grid_cost(valid, (32, 64), origin, bug), rel=1e-12), origin


def test_tile_origin_on_a_ringed_square():
    """A 2048 x 2048 catchment inside a one-cell no-data ring: the grid moves
    so that 32 tile columns cover the valid columns exactly (two of them
    general; the ring's columns fall in two tiles without valid cells), and
    the tiles over the top and bottom edges hold few rows."""
    from hipims_b200.fused import _first_valid_cell, tile_grid_cost, tile_origin

    n = 2048
    nodata = np.zeros((n + 2, n + 2), dtype=bool)
    nodata[0, :] = nodata[-1, :] = nodata[:, 0] = nodata[:, -1] = True
    mask = T.boundary_codes(nodata, default_bc=50)
    valid = mask > 0
    bug = _first_valid_cell(mask)
    o = tile_origin(valid, (32, 64), bug)
    assert o[1] == 63 and (n + 2 + o[0]) % 32 != 0
    assert tile_grid_cost(valid, (32, 64), o, bug) < 0.96 * tile_grid_cost(valid, (32, 64),
                                                                             (0, 0), bug)


def test_shifted_layout_views_and_offsets():
    """An instance on a shifted grid: the raster views, validity, bed and
    gather offsets are those of the catchment; the kernels' raster is larger
    by the shift, with no-data codes in the added rows and columns."""
    d = S.urban_catchment(100, seed=1, rain_mm_h=60.0)
    rng = np.random.default_rng(0)
    d["h"] = np.where(d["mask"] > 0, rng.uniform(0, 0.2, d["mask"].shape), 0.0)
    c = S.catchment_from(d)
    a = _Instance(c, torch.float32, "cpu", (32, 64))
    b = _Instance(c, torch.float32, "cpu", (32, 64), origin=(5, 11))
    assert (b.rows, b.cols) == (a.rows + 5, a.cols + 11)
    assert b.bug == (a.bug[0] + 5, a.bug[1] + 11)
    np.testing.assert_array_equal(b.valid, a.valid)
    np.testing.assert_array_equal(b.raster(b.h[0]).numpy(), a.raster(a.h[0]).numpy())
    zb = b.raster(b.z).double().numpy() + b.z_abs_offset
    v = d["mask"] > 0
    assert np.abs(zb[v] - d["z"][v]).max() < 1e-5
    code = b.code.numpy()
    PY, CPX = _lib.HB_PAD_Y, _lib.HB_CODE_PAD_X
    assert (code[PY:PY + 5, CPX:CPX + b.cols] >> 4 == _lib.HB_NODATA_CLASS).all()
    assert (code[PY:PY + b.rows, CPX:CPX + 11] >> 4 == _lib.HB_NODATA_CLASS).all()
    rr, cc = np.nonzero(v)
    sy, sx = b.origin
    off = (rr + PY + sy) * b.pitch + (cc + _lib.HB_PAD_X + sx)
    np.testing.assert_array_equal(b.h[0].numpy().ravel()[off], a.raster(a.h[0]).numpy()[v])
    with pytest.raises(ValueError):
        _Instance(c, torch.float32, "cpu", (32, 64), origin=(-1, 0))
