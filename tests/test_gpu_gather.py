"""Coupling gather: bit-exact depths at agent cells, in the reference's
compacted (row-major valid-cell) order."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def test_gather_matches_compacted_indexing(cuda):
    from hipims_b200 import ops, scenarios as S
    from hipims_b200.fused import FusedSolver
    from hipims_b200.scenarios import catchment_from

    d = S.urban_catchment(150, seed=2, rain_mm_h=300.0)
    fs = FusedSolver(catchment_from(d), dtype=torch.float32, device=cuda)
    fs.step(100)
    comp = fs.compacted()
    rng = np.random.default_rng(0)
    ids = np.sort(rng.choice(comp["h"].size, 500, replace=False))  # idx_target in compacted ids
    pos = np.argwhere(d["mask"] > 0)[ids]
    off = fs.cell_offsets(0, pos[:, 0], pos[:, 1])
    h, qx, qy = fs.current()
    gh, gu, gv = ops.gather(off, h, qx, qy, velocities=True)
    np.testing.assert_array_equal(gh.cpu().numpy().astype(np.float64), comp["h"][ids])
    wet = comp["h"][ids] > 1e-6
    u = np.where(wet, comp["qx"][ids] / np.where(wet, comp["h"][ids], 1), 0)
    np.testing.assert_allclose(gu.cpu().numpy(), u, rtol=1e-6, atol=1e-7)
