"""The plain FP64 GPU baseline (the reference's own kernels built for sm_100a,
driven by the Godunov loop) computes what the oracle computes: it is the
denominator of the fused step's speed-up, so it is checked like a product.
Only the boundary kinds the benchmark uses are exercised (walls and open
boundaries with id 0, default boundary tables)."""
import os
import sys

import numpy as np
import pytest
import torch

from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
from baseline import ref_gpu  # noqa: E402

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not ref_gpu.available(), reason="baseline/_ref not built")]


def run_reference_kernels(d, dev, steps):
    from hipims_b200.solver import Godunov

    g = Godunov(dev, d["dx"], d["cfl"], 1e30, secondOrder=True, firstTimeStep=d["first_dt"],
                tensorType=torch.float64, ops_impl=ref_gpu.RefGpuOps())
    g._export_enabled = False
    T = lambda a: torch.as_tensor(np.asarray(a, dtype=np.float64))
    mask = torch.as_tensor(np.asarray(d["mask"]))
    g.init__fluidField_tensor(mask, T(d["h"]), T(d["qx"]), T(d["qy"]),
                              T(np.asarray(d["z"]) + np.asarray(d["h"])), T(d["z"]), dev)
    g.set__frictionField_tensor(torch.as_tensor(np.atleast_1d(d["manning"]), device=dev), dev)
    g.set_landuse(mask, torch.as_tensor(np.asarray(d["landuse"])), dev)
    g.set_distributed_rainfall_station_Mask(mask, torch.zeros(mask.shape, dtype=torch.int16),
                                            dev)
    rain = d.get("rain")
    rain = np.array([[0.0, 0.0], [1e9, 0.0]]) if rain is None else np.asarray(rain)
    for _ in range(steps):
        g.addFlux()
        g.addStation_PrecipitationSource(rain, dev)
        g.time_friction_euler_update_cuda(dev)
    return g


@pytest.mark.parametrize("case,steps,atol", [("dam_break", 200, 1e-9), ("urban", 30, 1e-6)])
def test_reference_gpu_kernels_match_oracle(cuda, case, steps, atol):
    from hipims_b200 import scenarios as S

    d = S.dam_break(48) if case == "dam_break" else S.urban_catchment(64, dx=2.0, seed=4)
    sim = O.Sim(d, order=2)
    sim.run(steps)
    g = run_reference_kernels(d, cuda, steps)
    st = sim.state()
    assert g.t.item() == pytest.approx(st["t"], rel=1e-9)
    for k, x in (("h", g._h_internal), ("qx", g._qx_internal), ("qy", g._qy_internal)):
        np.testing.assert_allclose(x.cpu().numpy(), st[k], rtol=0, atol=atol, err_msg=k)
