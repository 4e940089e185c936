"""Small and degenerate catchments against the golden fixtures of the
reference's own kernels (tests/golden/edge_*.npz, made by make_golden.py):
a raster smaller than one tile, a single row, a single column, a dry
catchment without rain (dt grows tenfold per step up to the export clip) and
rain that starts after the first steps.

FP64: the fused step evaluates every face once where the reference evaluates
it from both cells, so the fields agree to round-off (1e-10 m) and the clock
(t, dt, export count) to 1e-12 relative.  FP32: the golden run's dt sequence
is replayed (the oracle reproduces the fixtures bit for bit) and depths agree
to 1e-4 m."""
import glob
import os

import numpy as np
import pytest
import torch

import make_golden as G
from oracle import oracle as O

pytestmark = pytest.mark.gpu

EDGE = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "edge_*.npz")))
IDS = [os.path.basename(p)[5:-4] for p in EDGE]


def solver(d, dtype, cuda, order, kernel="rows", **over):
    from hipims_b200.fused import FusedSolver
    from hipims_b200.scenarios import catchment_from

    c = catchment_from(d, export_step=d["export_step"], **over)
    return FusedSolver(c, dtype=dtype, tile=(32, 32), device=cuda, order=order, kernel=kernel)


def test_edge_fixtures_exist():
    assert len(EDGE) == 2 * len(G.EDGE_CASES)


@pytest.mark.parametrize("path", EDGE, ids=IDS)
def test_edge_case_fp64_matches_reference_kernels(cuda, path):
    d, order, exp = G.load_case(path)
    kernels = ["rows", "tasks"] if order == 2 else ["rows"]
    for kernel in kernels:
        fs = solver(d, torch.float64, cuda, order, kernel)
        fs.step(d["steps"])
        c = fs.controls()[0]
        assert c.step == int(exp["steps"]), kernel
        assert c.exports == int(exp["exports"]), kernel
        assert c.t == pytest.approx(float(exp["t"]), rel=1e-12), kernel
        assert c.dt == pytest.approx(float(exp["dt"]), rel=1e-12), kernel
        got = fs.compacted()
        err = {f: float(np.abs(got[f] - exp[f]).max()) for f in ("h", "qx", "qy", "h_max")}
        print(os.path.basename(path), kernel, err)
        assert max(err.values()) < 1e-10, (kernel, err)


@pytest.mark.parametrize("path", [p for p in EDGE if "_dry_" not in p],
                         ids=[i for i in IDS if not i.startswith("dry")])
def test_edge_case_fp32_with_replayed_dt(cuda, path):
    d, order, exp = G.load_case(path)
    sim = O.Sim(d, order=order, export_step=d["export_step"])
    dts = sim.run_record(d["steps"])
    np.testing.assert_array_equal(sim.state()["h"], exp["h"])
    fs = solver(d, torch.float32, cuda, order, dt_replay=dts)
    fs.step(d["steps"])
    got = fs.compacted()
    err = float(np.abs(got["h"] - exp["h"]).max())
    print(os.path.basename(path), "FP32 max|dh|", err)
    assert err <= 1e-4


def test_dry_catchment_stays_dry_and_clock_follows_reference(cuda):
    """No water and no rain: the state stays exactly zero in both precisions,
    and the clock takes the reference's dt sequence (x10 per step, then the
    export clip)."""
    path = [p for p in EDGE if "_dry_o2" in p][0]
    d, order, exp = G.load_case(path)
    sim = O.Sim(d, order=order, export_step=d["export_step"])
    want = sim.run_record(12)
    for dtype in (torch.float64, torch.float32):
        fs = solver(d, dtype, cuda, order)
        got = []
        for _ in range(12):
            t0 = fs.controls()[0].t
            fs.step(1)
            got.append(fs.controls()[0].t - t0)
        np.testing.assert_allclose(got, want, rtol=1e-12)
        st = fs.compacted()
        for f in ("h", "qx", "qy", "h_max"):
            assert not np.any(st[f]), f
