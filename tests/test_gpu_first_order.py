"""Fused 1st-order step: the reference's secondOrder = False scheme
(HC/fluxCal_jh_modified_surface_Kernel.cu, the coupled server's choice in
CHANS-HiPIMS_server.py) against the oracle's 1st-order scheme.

FP64: every face is evaluated once, so the match is to round-off (1e-10 m, as
for the 2nd-order fused step).  FP32: the oracle's dt sequence is replayed and
the north-star 1e-4 m holds over the early steps; the 1-D dam break keeps
qy = 0 exactly."""
import numpy as np
import pytest
import torch

import make_golden as G
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def catchment(d, **over):
    from hipims_b200.scenarios import catchment_from

    return catchment_from(d, **over)


def compare(fs, sim, k=0):
    got = fs.compacted(k)
    st = sim.state()
    return {f: float(np.abs(got[f] - st[f]).max()) for f in ("h", "qx", "qy", "h_max")}


def test_first_order_fp64_dam_break(cuda):
    from hipims_b200 import scenarios as S
    from hipims_b200.fused import FusedSolver

    d = S.dam_break(100)
    sim = O.Sim(d, order=1)
    sim.run(300)
    fs = FusedSolver(catchment(d), dtype=torch.float64, device=cuda, order=1)
    fs.step(300)
    c = fs.controls()[0]
    assert c.step == 300
    assert c.t == pytest.approx(sim.t, rel=1e-10)
    err = compare(fs, sim)
    assert max(err.values()) < 1e-9, err


def test_first_order_fp64_channel(cuda):
    """H_GIVEN inflow, OPEN outflow, walls, to t = 3 s (the reference's own
    1st-order scheme goes unstable on this case near t = 4.9 s)."""
    from hipims_b200 import scenarios as S
    from hipims_b200.fused import FusedSolver

    d = S.channel()
    sim = O.Sim(d, order=1)
    n = sim.run(100000, 3.0)
    fs = FusedSolver(catchment(d, t_end=3.0), dtype=torch.float64, device=cuda, order=1)
    fs.step(n + 5)
    c = fs.controls()[0]
    assert c.step == n and c.halted
    err = compare(fs, sim)
    assert max(err.values()) < 1e-10, err


@pytest.mark.parametrize("seed", [1, 2])
def test_first_order_fp64_mixed_boundaries_with_fall(cuda, seed):
    """Every ghost type including FALL (type 9, 1st order only), an interior
    hole, wet/dry cells, rain and export clips."""
    from hipims_b200.fused import FusedSolver

    d = G.mixed_bc_case(300 + seed, 1)
    d.pop("rain_mask")
    d["rain"] = np.array([[0.0, 2e-4], [1.0, 5e-4], [10.0, 0.0]])
    sim = O.Sim(d, order=1, export_step=0.75)
    fs = FusedSolver(catchment(d, export_step=0.75), dtype=torch.float64, device=cuda, order=1)
    done = 0
    for k, tol in ((6, 1e-12), (60, 1e-3)):
        sim.run(k - done)
        fs.step(k - done)
        done = k
        c = fs.controls()[0]
        assert c.exports == sim.g.exports and c.t == pytest.approx(sim.t, rel=max(tol, 1e-12))
        err = compare(fs, sim)
        print("1st-order mixed bc FP64 fused vs oracle after", k, "steps:", err)
        assert (max(err.values()) if k <= 6 else err["h"]) < tol, (k, err)


@pytest.mark.parametrize("tile,minb", [((32, 32), 5), ((32, 64), 0)])
def test_first_order_fp32_dam_break(cuda, tile, minb):
    """256 x 256 dam break in FP32 against the FP64 oracle at the same
    simulated times; uniform along y, so qy stays exactly 0.  Both step
    kernels: one cell per lane (32 x 32) and two (32 x 64)."""
    from hipims_b200 import scenarios as S
    from hipims_b200.fused import FusedSolver

    d = S.dam_break(256)
    sim = O.Sim(d, order=1)
    dts = sim.run_record(200)
    ref = O.Sim(d, order=1)
    ref.run(200)
    fs = FusedSolver(catchment(d, dt_replay=dts), dtype=torch.float32, device=cuda, order=1,
                     tile=tile, minb=minb)
    fs.step(200)
    got = fs.compacted()
    err = float(np.abs(got["h"] - ref.h).max())
    print("1st-order FP32 dam break", tile, "200 steps, max|dh|", err)
    assert np.abs(got["qy"]).max() == 0.0
    assert err <= 1e-4


@pytest.mark.parametrize("tile", [(32, 32), (32, 64)])
def test_first_order_fp32_urban_rain(cuda, tile):
    """Rain on the urban DEM (buildings, two Manning zones, open ring, dry
    start) in FP32 against the FP64 oracle at the same simulated times."""
    from hipims_b200 import scenarios as S
    from hipims_b200.fused import FusedSolver

    d = S.urban_catchment(192, dx=2.0, seed=3, rain_mm_h=200.0)
    sim = O.Sim(d, order=1)
    dts = sim.run_record(25)
    ref = O.Sim(d, order=1)
    ref.run(25)
    fs = FusedSolver(catchment(d, dt_replay=dts), dtype=torch.float32, device=cuda, order=1,
                     tile=tile)
    fs.step(25)
    err = float(np.abs(fs.compacted()["h"] - ref.h).max())
    print("1st-order urban FP32", tile, "vs FP64 oracle after 25 steps, max|dh|", err)
    assert err <= 2e-4


def test_first_order_strips_reproduce_the_undivided_run(cuda):
    from hipims_b200 import scenarios as S
    from hipims_b200.fused import FusedSolver
    from hipims_b200.strips import StripSolver

    d = S.urban_catchment(192, dx=2.0, seed=8, rain_mm_h=120.0)
    c = S.catchment_from(d)
    one = FusedSolver(c, dtype=torch.float32, device=cuda, order=1, origin=(0, 0))
    st = StripSolver(c, 3, dtype=torch.float32, device=cuda, order=1)
    one.step(40)
    st.step(40)
    a, b = one.state(), st.state()
    for f in ("h", "qx", "qy", "h_max"):
        assert torch.equal(a[f], b[f]), f


@pytest.mark.parametrize("seed", [1, 2])
@pytest.mark.parametrize("tile", [(32, 32), (32, 64)])
def test_first_order_fp32_mixed_boundaries_with_fall(cuda, seed, tile):
    """FP32 1st order on every ghost type FALL included, station rain off,
    against the FP64 oracle with its dt sequence replayed (both kernels)."""
    from hipims_b200.fused import FusedSolver

    d = G.mixed_bc_case(200 + seed, 1)
    d.pop("rain_mask")
    d["rain"] = np.array([[0.0, 2e-4], [1.0, 5e-4], [10.0, 0.0]])
    sim = O.Sim(d, order=1)
    dts = sim.run_record(8)
    fs = FusedSolver(catchment(d, dt_replay=dts), dtype=torch.float32, device=cuda, order=1,
                     tile=tile)
    fs.step(8)
    err = compare(fs, sim)
    print("1st-order mixed bc FP32", tile, "vs oracle after 8 steps:", err)
    assert err["h"] < 1e-4 and err["qx"] < 1e-4 and err["qy"] < 1e-4, err
